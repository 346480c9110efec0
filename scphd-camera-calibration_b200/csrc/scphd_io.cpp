// File input/output around the filter step: configuration files in libconfig syntax,
// MATLAB level-5 MAT files (measurement cells in, filter state out).  Host code only;
// the result writer reads the filter through the library's C ABI.
#include "scphd_io.h"

#include <zlib.h>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

__attribute__((visibility("hidden"))) scphd_status scphd_fail_internal(scphd_status st, const char* msg);

namespace {

scphd_status fail(scphd_status st, const std::string& m) { return scphd_fail_internal(st, m.c_str()); }

// ======================================================================= configuration
// A setting is a number, boolean, string, group or list; groups keep their keys.
struct Setting {
    enum Kind { NUM, BOOL, STR, GROUP, LIST } kind = NUM;
    double num = 0;
    bool b = false;
    std::string str;
    std::map<std::string, std::unique_ptr<Setting>> group;
    std::vector<std::unique_ptr<Setting>> list;
    int line = 0;
};

class ConfigParser {
  public:
    ConfigParser(const std::string& text, const std::string& file) : s_(text), file_(file) {}

    bool parse(Setting& root, std::string& err) {
        root.kind = Setting::GROUP;
        if (!settings(root, '\0', err)) return false;
        return true;
    }

  private:
    const std::string& s_;
    std::string file_;
    size_t i_ = 0;
    int line_ = 1;

    std::string where() const { return file_ + ":" + std::to_string(line_); }

    void skip() {   // whitespace and comments
        while (i_ < s_.size()) {
            char c = s_[i_];
            if (c == '\n') { ++line_; ++i_; }
            else if (isspace((unsigned char)c)) ++i_;
            else if (c == '#' || (c == '/' && i_ + 1 < s_.size() && s_[i_ + 1] == '/')) {
                while (i_ < s_.size() && s_[i_] != '\n') ++i_;
            } else if (c == '/' && i_ + 1 < s_.size() && s_[i_ + 1] == '*') {
                i_ += 2;
                while (i_ + 1 < s_.size() && !(s_[i_] == '*' && s_[i_ + 1] == '/')) {
                    if (s_[i_] == '\n') ++line_;
                    ++i_;
                }
                i_ += 2;
            } else break;
        }
    }

    bool name(std::string& out) {
        skip();
        size_t b = i_;
        if (i_ < s_.size() && (isalpha((unsigned char)s_[i_]) || s_[i_] == '*')) {
            ++i_;
            while (i_ < s_.size() && (isalnum((unsigned char)s_[i_]) || s_[i_] == '_' || s_[i_] == '-' || s_[i_] == '*'))
                ++i_;
        }
        out = s_.substr(b, i_ - b);
        return !out.empty();
    }

    // settings until `close` ('}' of a group, or end of text)
    bool settings(Setting& grp, char close, std::string& err) {
        while (true) {
            skip();
            if (i_ >= s_.size()) {
                if (close) { err = where() + ": missing '}'"; return false; }
                return true;
            }
            if (close && s_[i_] == close) { ++i_; return true; }
            std::string key;
            if (!name(key)) { err = where() + ": expected a setting name"; return false; }
            skip();
            if (i_ >= s_.size() || (s_[i_] != '=' && s_[i_] != ':')) {
                err = where() + ": expected '=' or ':' after " + key;
                return false;
            }
            ++i_;
            std::unique_ptr<Setting> v(new Setting());
            if (!value(*v, err)) return false;
            skip();
            if (i_ < s_.size() && (s_[i_] == ';' || s_[i_] == ',')) ++i_;
            grp.group[key] = std::move(v);
        }
    }

    bool value(Setting& v, std::string& err) {
        skip();
        v.line = line_;
        if (i_ >= s_.size()) { err = where() + ": missing value"; return false; }
        char c = s_[i_];
        if (c == '{') {
            ++i_;
            v.kind = Setting::GROUP;
            return settings(v, '}', err);
        }
        if (c == '[' || c == '(') {
            const char close = c == '[' ? ']' : ')';
            ++i_;
            v.kind = Setting::LIST;
            while (true) {
                skip();
                if (i_ < s_.size() && s_[i_] == close) { ++i_; return true; }
                std::unique_ptr<Setting> e(new Setting());
                if (!value(*e, err)) return false;
                v.list.push_back(std::move(e));
                skip();
                if (i_ < s_.size() && s_[i_] == ',') ++i_;
            }
        }
        if (c == '"') {
            v.kind = Setting::STR;
            ++i_;
            while (i_ < s_.size() && s_[i_] != '"') {
                if (s_[i_] == '\\' && i_ + 1 < s_.size()) ++i_;
                v.str += s_[i_++];
            }
            if (i_ >= s_.size()) { err = where() + ": unterminated string"; return false; }
            ++i_;
            return true;
        }
        size_t b = i_;
        while (i_ < s_.size() && !isspace((unsigned char)s_[i_]) && s_[i_] != ';' && s_[i_] != ',' &&
               s_[i_] != '}' && s_[i_] != ']' && s_[i_] != ')' && s_[i_] != '#')
            ++i_;
        std::string tok = s_.substr(b, i_ - b);
        std::string low;
        for (char ch : tok) low += (char)tolower((unsigned char)ch);
        if (low == "true" || low == "false") {
            v.kind = Setting::BOOL;
            v.b = low == "true";
            v.num = v.b ? 1 : 0;
            return true;
        }
        if (!low.empty() && low.back() == 'l') low.pop_back();   // 64-bit integer suffix
        if (!low.empty() && low.back() == 'l') low.pop_back();
        char* end = nullptr;
        const double d = (low.size() > 2 && low[0] == '0' && low[1] == 'x') ? (double)strtoull(low.c_str(), &end, 16)
                                                                            : strtod(low.c_str(), &end);
        if (tok.empty() || !end || *end != '\0') {
            err = where() + ": cannot read value '" + tok + "'";
            return false;
        }
        v.kind = Setting::NUM;
        v.num = d;
        return true;
    }
};

const Setting* lookup(const Setting& root, const std::string& path) {
    const Setting* cur = &root;
    size_t b = 0;
    while (b <= path.size()) {
        size_t e = path.find('.', b);
        if (e == std::string::npos) e = path.size();
        if (cur->kind != Setting::GROUP) return nullptr;
        auto it = cur->group.find(path.substr(b, e - b));
        if (it == cur->group.end()) return nullptr;
        cur = it->second.get();
        b = e + 1;
    }
    return cur;
}

// a numeric setting, if present; false (with err) if present but not numeric
bool num(const Setting& root, const std::string& key, double& out, bool& found, std::string& err) {
    const Setting* s = lookup(root, key);
    found = s != nullptr;
    if (!s) return true;
    if (s->kind != Setting::NUM && s->kind != Setting::BOOL) {
        err = "setting " + key + " (line " + std::to_string(s->line) + ") is not a number";
        return false;
    }
    out = s->num;
    return true;
}

// ======================================================================= MAT level 5
enum : uint32_t {
    miINT8 = 1, miUINT8 = 2, miINT16 = 3, miUINT16 = 4, miINT32 = 5, miUINT32 = 6, miSINGLE = 7,
    miDOUBLE = 9, miINT64 = 12, miUINT64 = 13, miMATRIX = 14, miCOMPRESSED = 15, miUTF8 = 16
};
enum : uint8_t { mxCELL = 1, mxSTRUCT = 2, mxDOUBLE = 6, mxSINGLE = 7, mxINT8 = 8, mxUINT64 = 15 };

struct Reader {
    const uint8_t* p;
    size_t n, at = 0;
    bool ok = true;
    bool tag(uint32_t& type, uint32_t& bytes, const uint8_t*& data) {
        if (at + 8 > n) return ok = false;
        uint32_t w0, w1;
        memcpy(&w0, p + at, 4);
        memcpy(&w1, p + at + 4, 4);
        if (w0 >> 16) {   // small data element: 2-byte size, 2-byte type, 4 bytes of data
            type = w0 & 0xffff;
            bytes = w0 >> 16;
            data = p + at + 4;
            at += 8;
            return bytes <= 4 || (ok = false);
        }
        type = w0;
        bytes = w1;
        if (at + 8 + (size_t)bytes > n) return ok = false;
        data = p + at + 8;
        // elements are padded to 8 bytes, except compressed ones
        at += 8 + (type == 15 ? (size_t)bytes : (((size_t)bytes + 7) & ~(size_t)7));
        if (at > n) at = n;   // the last element may end without padding
        return true;
    }
};

size_t type_size(uint32_t t) {
    switch (t) {
        case miINT8: case miUINT8: case miUTF8: return 1;
        case miINT16: case miUINT16: return 2;
        case miINT32: case miUINT32: case miSINGLE: return 4;
        case miDOUBLE: case miINT64: case miUINT64: return 8;
        default: return 0;
    }
}

double elem(uint32_t t, const uint8_t* d, size_t i) {
    switch (t) {
        case miINT8: return (double)((const int8_t*)d)[i];
        case miUINT8: return (double)d[i];
        case miINT16: { int16_t v; memcpy(&v, d + 2 * i, 2); return v; }
        case miUINT16: { uint16_t v; memcpy(&v, d + 2 * i, 2); return v; }
        case miINT32: { int32_t v; memcpy(&v, d + 4 * i, 4); return v; }
        case miUINT32: { uint32_t v; memcpy(&v, d + 4 * i, 4); return v; }
        case miSINGLE: { float v; memcpy(&v, d + 4 * i, 4); return v; }
        case miDOUBLE: { double v; memcpy(&v, d + 8 * i, 8); return v; }
        case miINT64: { int64_t v; memcpy(&v, d + 8 * i, 8); return (double)v; }
        case miUINT64: { uint64_t v; memcpy(&v, d + 8 * i, 8); return (double)v; }
        default: return NAN;
    }
}

// A parsed array: numeric (real part, column-major) or cell (children).
struct Array {
    uint8_t cls = 0;
    std::vector<int32_t> dims;
    std::string name;
    std::vector<double> re;
    std::vector<Array> cells;
};

bool parse_matrix(const uint8_t* d, size_t n, Array& a, std::string& err, int depth = 0) {
    if (depth > 16) { err = "MAT: nesting too deep"; return false; }
    Reader r{d, n};
    uint32_t t, b;
    const uint8_t* x;
    if (!r.tag(t, b, x) || t != miUINT32 || b < 4) { err = "MAT: bad array flags"; return false; }
    uint32_t flags;
    memcpy(&flags, x, 4);
    a.cls = flags & 0xff;
    const bool complex = (flags >> 11) & 1;
    if (!r.tag(t, b, x) || t != miINT32) { err = "MAT: bad dimensions"; return false; }
    a.dims.resize(b / 4);
    size_t count = 1;
    for (size_t k = 0; k < a.dims.size(); ++k) {
        memcpy(&a.dims[k], x + 4 * k, 4);
        if (a.dims[k] < 0) { err = "MAT: negative dimension"; return false; }
        count *= (size_t)a.dims[k];
    }
    if (count > ((size_t)1 << 32)) { err = "MAT: array too large"; return false; }
    if (!r.tag(t, b, x)) { err = "MAT: bad name"; return false; }
    a.name.assign((const char*)x, b);
    if (a.cls == mxCELL) {
        a.cells.resize(count);
        for (size_t k = 0; k < count; ++k) {
            if (!r.tag(t, b, x) || t != miMATRIX) { err = "MAT: bad cell element"; return false; }
            if (b == 0) continue;   // empty cell
            if (!parse_matrix(x, b, a.cells[k], err, depth + 1)) return false;
        }
        return true;
    }
    if (a.cls >= mxDOUBLE && a.cls <= mxUINT64) {
        if (!r.tag(t, b, x)) { err = "MAT: bad real part"; return false; }
        const size_t es = type_size(t);
        if (!es || (size_t)b / es < count) { err = "MAT: unsupported numeric storage"; return false; }
        a.re.resize(count);
        for (size_t k = 0; k < count; ++k) a.re[k] = elem(t, x, k);
        (void)complex;   // imaginary parts are ignored
        return true;
    }
    return true;   // structs, objects, characters, sparse: kept as opaque (no data)
}

bool inflate_all(const uint8_t* d, size_t n, std::vector<uint8_t>& out) {
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) return false;
    zs.next_in = const_cast<Bytef*>(d);
    zs.avail_in = (uInt)n;
    out.resize(n * 4 + 1024);
    int rc;
    do {
        if (zs.total_out >= out.size()) out.resize(out.size() * 2);
        zs.next_out = out.data() + zs.total_out;
        zs.avail_out = (uInt)(out.size() - zs.total_out);
        rc = inflate(&zs, Z_NO_FLUSH);
    } while (rc == Z_OK);
    out.resize(zs.total_out);
    inflateEnd(&zs);
    return rc == Z_STREAM_END;
}

// find and parse top-level variable `var`
bool read_variable(const std::string& path, const std::string& var, Array& a, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return false; }
    std::vector<uint8_t> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    if (buf.size() < 128) { err = path + ": not a MAT file"; return false; }
    if (buf[126] != 'I' || buf[127] != 'M') { err = path + ": not a little-endian level-5 MAT file"; return false; }
    Reader r{buf.data(), buf.size(), 128};
    while (r.at + 8 <= r.n) {
        uint32_t t, b;
        const uint8_t* x;
        if (!r.tag(t, b, x)) break;
        std::vector<uint8_t> inflated;
        const uint8_t* md = x;
        size_t mn = b;
        if (t == miCOMPRESSED) {
            if (!inflate_all(x, b, inflated)) { err = path + ": corrupt compressed element"; return false; }
            Reader ir{inflated.data(), inflated.size()};
            const uint8_t* y;
            if (!ir.tag(t, b, y)) continue;
            md = y;
            mn = b;
        }
        if (t != miMATRIX) continue;
        // the name comes after the flags and the dimensions: peek it before a full parse
        Reader pr{md, mn};
        uint32_t tt, bb;
        const uint8_t* y;
        if (!pr.tag(tt, bb, y) || !pr.tag(tt, bb, y) || !pr.tag(tt, bb, y)) continue;
        if (std::string((const char*)y, bb) != var) continue;
        return parse_matrix(md, mn, a, err);
    }
    err = path + ": no variable " + var;
    return false;
}

class MatWriter {
  public:
    std::vector<uint8_t> buf;
    MatWriter() {
        std::string h = "MATLAB 5.0 MAT-file, written by libscphd_b200";
        h.resize(116, ' ');
        buf.assign(h.begin(), h.end());
        buf.resize(124, 0);   // no subsystem data
        put16(0x0100);
        buf.push_back('I');
        buf.push_back('M');
    }
    // a real matrix (column-major data) as a top-level variable or a struct field
    void matrix(std::vector<uint8_t>& out, const std::string& name, const std::vector<int32_t>& dims,
                const double* data) {
        std::vector<uint8_t> body;
        header(body, mxDOUBLE, dims, name);
        size_t count = 1;
        for (int32_t d : dims) count *= (size_t)d;
        element(body, miDOUBLE, data, count * 8);
        element(out, miMATRIX, body.data(), body.size());
    }
    // a struct array; fields[element][field] are already-encoded miMATRIX bodies
    void structure(std::vector<uint8_t>& out, const std::string& name, const std::vector<int32_t>& dims,
                   const std::vector<std::string>& fields, const std::vector<std::vector<std::vector<uint8_t>>>& vals) {
        std::vector<uint8_t> body;
        header(body, mxSTRUCT, dims, name);
        const int32_t len = 32;
        // field name length: a small data element
        uint32_t w0 = (4u << 16) | miINT32;
        append(body, &w0, 4);
        append(body, &len, 4);
        std::vector<char> names(fields.size() * len, 0);
        for (size_t k = 0; k < fields.size(); ++k) memcpy(names.data() + k * len, fields[k].c_str(), fields[k].size());
        element(body, miINT8, names.data(), names.size());
        for (const auto& e : vals)
            for (const auto& v : e) body.insert(body.end(), v.begin(), v.end());
        element(out, miMATRIX, body.data(), body.size());
    }
    bool save(const std::string& path, std::string& err) {
        FILE* f = fopen(path.c_str(), "wb");
        if (!f) { err = "cannot write " + path; return false; }
        const bool ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
        if (fclose(f) != 0 || !ok) { err = "write failed: " + path; return false; }
        return true;
    }

  private:
    void put16(uint16_t v) { append(buf, &v, 2); }
    static void append(std::vector<uint8_t>& o, const void* p, size_t n) {
        const uint8_t* c = (const uint8_t*)p;
        o.insert(o.end(), c, c + n);
    }
    static void element(std::vector<uint8_t>& o, uint32_t type, const void* p, size_t n) {
        uint32_t t[2] = {type, (uint32_t)n};
        append(o, t, 8);
        append(o, p, n);
        o.resize(o.size() + ((8 - n % 8) % 8), 0);
    }
    static void header(std::vector<uint8_t>& o, uint8_t cls, const std::vector<int32_t>& dims, const std::string& name) {
        uint32_t flags[2] = {cls, 0};
        element(o, miUINT32, flags, 8);
        element(o, miINT32, dims.data(), dims.size() * 4);
        element(o, miINT8, name.data(), name.size());
    }
};

std::vector<uint8_t> field_matrix(MatWriter& w, const std::vector<int32_t>& dims, const double* data) {
    std::vector<uint8_t> v;
    w.matrix(v, "", dims, data);
    return v;
}

// packed lower 6 x 6 -> full column-major
void unpack6(const double* p, double* full) {
    for (int a = 0; a < 6; ++a)
        for (int c = 0; c <= a; ++c) {
            const double v = p[a * (a + 1) / 2 + c];
            full[a + 6 * c] = v;
            full[c + 6 * a] = v;
        }
}

}  // namespace

extern "C" {

scphd_status scphd_config_from_file(const char* path, scphd_config* cfg, scphd_run_options* opts) {
    if (!path || !cfg || !opts) return fail(SCPHD_ERR_INVALID, "null argument");
    std::ifstream f(path);
    if (!f) return fail(SCPHD_ERR_INVALID, std::string("cannot open ") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    Setting root;
    std::string err;
    ConfigParser parser(text, path);
    if (!parser.parse(root, err)) return fail(SCPHD_ERR_INVALID, err);
    bool found = false;
    double v = 0;
#define NUMKEY(key, dst, conv)                                                     \
    do {                                                                           \
        if (!num(root, key, v, found, err)) return fail(SCPHD_ERR_INVALID, err);   \
        if (found) dst = conv(v);                                                  \
    } while (0)
#define ASIS(x) (x)
#define I32(x) ((int32_t)llround(x))
    NUMKEY("n_particles", cfg->n_parents, I32);
    NUMKEY("particles_per_feature", cfg->particles_per_feature, I32);
    NUMKEY("min_weight", cfg->min_weight, ASIS);
    NUMKEY("min_separation", cfg->min_separation, ASIS);
    NUMKEY("min_neff", cfg->min_neff, ASIS);
    NUMKEY("ps", cfg->ps, ASIS);
    static const char* axes[6] = {"x", "y", "z", "vx", "vy", "vz"};
    static const char* groups[2] = {"cartesian", "angular"};
    for (int g = 0; g < 2; ++g)
        for (int k = 0; k < 6; ++k) {
            const std::string base = std::string("prior.") + groups[g] + "." + axes[k];
            const int q = 6 * g + k;
            double a = 0, b = 0, mean = 0, sd = 0;
            bool fa, fb, fm, fs;
            if (!num(root, base + ".a", a, fa, err) || !num(root, base + ".b", b, fb, err) ||
                !num(root, base + ".mean", mean, fm, err) || !num(root, base + ".std", sd, fs, err))
                return fail(SCPHD_ERR_INVALID, err);
            if (fa != fb) return fail(SCPHD_ERR_INVALID, "prior " + base + " needs both a and b");
            if (fa) {
                cfg->prior_a[q] = a;
                cfg->prior_b[q] = b;
            } else if (fm) {
                cfg->prior_a[q] = mean - (fs ? sd : 0.0);
                cfg->prior_b[q] = mean + (fs ? sd : 0.0);
            }
        }
    NUMKEY("camera_motion_model.cartesian.ax", cfg->cam_std[0], ASIS);
    NUMKEY("camera_motion_model.cartesian.ay", cfg->cam_std[1], ASIS);
    NUMKEY("camera_motion_model.cartesian.az", cfg->cam_std[2], ASIS);
    NUMKEY("camera_motion_model.angular.ax", cfg->cam_std[3], ASIS);
    NUMKEY("camera_motion_model.angular.ay", cfg->cam_std[4], ASIS);
    NUMKEY("camera_motion_model.angular.az", cfg->cam_std[5], ASIS);
    NUMKEY("feature_motion_model.ax", cfg->feat_std[0], ASIS);
    NUMKEY("feature_motion_model.ay", cfg->feat_std[1], ASIS);
    NUMKEY("feature_motion_model.az", cfg->feat_std[2], ASIS);
    NUMKEY("measurement_model.fx", cfg->fx, ASIS);
    NUMKEY("measurement_model.fy", cfg->fy, ASIS);
    NUMKEY("measurement_model.u0", cfg->u0, ASIS);
    NUMKEY("measurement_model.v0", cfg->v0, ASIS);
    NUMKEY("measurement_model.std_u", cfg->std_u, ASIS);
    NUMKEY("measurement_model.std_v", cfg->std_v, ASIS);
    NUMKEY("measurement_model.std_d", cfg->std_d, ASIS);
    NUMKEY("measurement_model.pd", cfg->pd, ASIS);
    double lambda = 0;
    bool flam = false;
    if (!num(root, "measurement_model.lambda", lambda, flam, err)) return fail(SCPHD_ERR_INVALID, err);
    if (flam) {
        if (!(cfg->v0 > 0)) return fail(SCPHD_ERR_INVALID, "measurement_model.lambda needs v0 > 0");
        cfg->kappa = lambda / ((2 * cfg->v0) * (2 * cfg->v0));
    }
    NUMKEY("measurement_model.kappa", cfg->kappa, ASIS);
    NUMKEY("birth.w0", cfg->w0, ASIS);
    NUMKEY("birth.d0", cfg->d0, ASIS);
    NUMKEY("birth.vu0", cfg->vu0, ASIS);
    NUMKEY("birth.vv0", cfg->vv0, ASIS);
    NUMKEY("birth.vd0", cfg->vd0, ASIS);
    NUMKEY("birth.var_d0", cfg->var_d0, ASIS);
    NUMKEY("birth.var_vu0", cfg->var_vu0, ASIS);
    NUMKEY("birth.var_vv0", cfg->var_vv0, ASIS);
    NUMKEY("birth.var_vd0", cfg->var_vd0, ASIS);
    NUMKEY("max_steps", opts->max_steps, I32);
    NUMKEY("slam", opts->slam, I32);
    NUMKEY("save_all_maps", opts->save_all_maps, I32);
    NUMKEY("verbosity", opts->verbosity, I32);
    NUMKEY("max_gaussians", cfg->max_gaussians, I32);
    NUMKEY("max_measurements", cfg->max_measurements, I32);
    NUMKEY("max_survivors", cfg->max_survivors, I32);
    NUMKEY("meas_dim", cfg->meas_dim, I32);
    NUMKEY("device", cfg->device, I32);
    NUMKEY("baseline", cfg->baseline, ASIS);
    NUMKEY("seed", cfg->seed, (uint64_t));
    if (const Setting* p = lookup(root, "precision")) {
        if (p->kind == Setting::STR) {
            if (p->str == "fp32") cfg->precision = SCPHD_FP32;
            else if (p->str == "fp64") cfg->precision = SCPHD_FP64;
            else return fail(SCPHD_ERR_INVALID, "precision must be \"fp32\" or \"fp64\"");
        } else if (p->kind == Setting::NUM) {
            cfg->precision = (int32_t)p->num;
        }
    }
#undef NUMKEY
#undef ASIS
#undef I32
    return SCPHD_OK;
}

scphd_status scphd_read_mat_frames(const char* path, const char* var, int32_t* n_frames, int32_t* rows,
                                   int32_t* sizes, double* data, int64_t data_capacity) {
    if (!path || !var || !n_frames || !rows) return fail(SCPHD_ERR_INVALID, "null argument");
    Array a;
    std::string err;
    if (!read_variable(path, var, a, err)) return fail(SCPHD_ERR_INVALID, err);
    if (a.cls != mxCELL) return fail(SCPHD_ERR_INVALID, std::string(var) + " is not a cell array");
    int32_t r = 0;
    for (const Array& c : a.cells) {
        if (c.dims.empty() || c.re.empty()) continue;   // empty frames
        if (c.dims.size() != 2 || (c.dims[0] != 2 && c.dims[0] != 3))
            return fail(SCPHD_ERR_INVALID, std::string(var) + ": frames must be 2 x n or 3 x n matrices");
        if (r && c.dims[0] != r) return fail(SCPHD_ERR_INVALID, std::string(var) + ": frames differ in rows");
        r = c.dims[0];
    }
    *n_frames = (int32_t)a.cells.size();
    *rows = r ? r : 2;
    if (!sizes && !data) return SCPHD_OK;
    if (!sizes || !data) return fail(SCPHD_ERR_INVALID, "sizes and data go together");
    int64_t at = 0;
    for (size_t k = 0; k < a.cells.size(); ++k) {
        const Array& c = a.cells[k];
        const int32_t n = c.re.empty() ? 0 : c.dims[1];
        sizes[k] = n;
        if (at + (int64_t)(*rows) * n > data_capacity) return fail(SCPHD_ERR_CAPACITY, "data buffer too small");
        for (int32_t q = 0; q < *rows; ++q)
            for (int32_t i = 0; i < n; ++i) data[at + (int64_t)q * n + i] = c.re[(size_t)i * (*rows) + q];
        at += (int64_t)(*rows) * n;
    }
    return SCPHD_OK;
}

scphd_status scphd_write_mat_arrays(const char* path, int32_t n, const char* const* names, const int32_t* rows,
                                    const int32_t* cols, const double* const* data) {
    if (!path || n < 0 || (n > 0 && (!names || !rows || !cols || !data))) return fail(SCPHD_ERR_INVALID, "null argument");
    MatWriter w;
    for (int32_t k = 0; k < n; ++k) {
        if (!names[k] || rows[k] < 0 || cols[k] < 0) return fail(SCPHD_ERR_INVALID, "bad array description");
        w.matrix(w.buf, names[k], {rows[k], cols[k]}, data[k]);
    }
    std::string err;
    if (!w.save(path, err)) return fail(SCPHD_ERR_INVALID, err);
    return SCPHD_OK;
}

scphd_status scphd_write_mat(scphd_filter* f, const char* path, int32_t save_all_maps) {
    if (!f || !path) return fail(SCPHD_ERR_INVALID, "null argument");
    // the configuration the filter was created with
    scphd_config cfg;
    scphd_status st = scphd_get_config(f, &cfg);
    if (st != SCPHD_OK) return st;
    const int N = cfg.n_parents, P = cfg.particles_per_feature;
    std::vector<double> states((size_t)N * 12), lw(N);
    if ((st = scphd_get_particles(f, states.data(), lw.data())) != SCPHD_OK) return st;
    MatWriter w;
    // particles: 12 x N column-major = the N x 12 row-major state array
    w.matrix(w.buf, "particles", {12, N}, states.data());
    int pmap = 0;
    double mx = -INFINITY;
    for (int p = 0; p < N; ++p)
        if (lw[p] > mx) { mx = lw[p]; pmap = p; }
    std::vector<double> lin(N);
    double tot = 0;
    for (int p = 0; p < N; ++p) tot += (lin[p] = std::exp(lw[p] - mx));
    for (int p = 0; p < N; ++p) lin[p] /= tot;
    w.matrix(w.buf, "weights", {N, 1}, lin.data());
    w.matrix(w.buf, "log_weights", {N, 1}, lw.data());
    // features: the MAP parent's map, clouds in the world frame
    std::vector<int32_t> sizes(N);
    if ((st = scphd_get_map_sizes(f, sizes.data())) != SCPHD_OK) return st;
    const int G = sizes[pmap];
    std::vector<double> fw(G), xyz((size_t)G * 6 * P), om((size_t)G * P), parts((size_t)6 * G * P);
    if (G > 0) {
        if ((st = scphd_get_map_weights(f, pmap, fw.data())) != SCPHD_OK) return st;
        if ((st = scphd_get_map_clouds(f, pmap, xyz.data(), om.data())) != SCPHD_OK) return st;
        for (int g = 0; g < G; ++g)
            for (int s = 0; s < P; ++s)
                for (int a = 0; a < 6; ++a) parts[((size_t)g * P + s) * 6 + a] = xyz[((size_t)g * 6 + a) * P + s];
    }
    {
        std::vector<std::vector<std::vector<uint8_t>>> vals(1);
        if (G > 0) {
            vals[0].push_back(field_matrix(w, {G, 1}, fw.data()));
            vals[0].push_back(field_matrix(w, {6, G * P}, parts.data()));
        } else {
            vals[0].push_back(field_matrix(w, {0, 0}, nullptr));
            vals[0].push_back(field_matrix(w, {0, 0}, nullptr));
        }
        w.structure(w.buf, "features", {1, 1}, {"weights", "particles"}, vals);
    }
    if (save_all_maps) {
        for (int which = 0; which < 2; ++which) {
            const int width = which == SCPHD_MIX_FITTED ? 29 : 28, off = which == SCPHD_MIX_FITTED ? 2 : 1;
            std::vector<std::vector<std::vector<uint8_t>>> vals(N);
            std::vector<double> rowsbuf;
            for (int p = 0; p < N; ++p) {
                int32_t cnt = 0;
                if ((st = scphd_get_mixture(f, which, p, nullptr, &cnt)) != SCPHD_OK) return st;
                rowsbuf.assign((size_t)cnt * width, 0.0);
                if (cnt && (st = scphd_get_mixture(f, which, p, rowsbuf.data(), &cnt)) != SCPHD_OK) return st;
                std::vector<double> wv(cnt), mv((size_t)6 * cnt), cv((size_t)36 * cnt);
                for (int i = 0; i < cnt; ++i) {
                    const double* r = rowsbuf.data() + (size_t)i * width;
                    wv[i] = r[0];
                    for (int a = 0; a < 6; ++a) mv[(size_t)i * 6 + a] = r[off + a];
                    unpack6(r + off + 6, cv.data() + (size_t)i * 36);
                }
                vals[p].push_back(field_matrix(w, {1, cnt}, wv.data()));
                vals[p].push_back(field_matrix(w, {6, cnt}, mv.data()));
                vals[p].push_back(field_matrix(w, {6, 6, cnt}, cv.data()));
            }
            w.structure(w.buf, which == SCPHD_MIX_FITTED ? "features_predicted" : "features_merged", {N, 1},
                        {"weights", "means", "covs"}, vals);
        }
        w.matrix(w.buf, "features_updated", {0, 0}, nullptr);
    }
    std::string err;
    if (!w.save(path, err)) return fail(SCPHD_ERR_INVALID, err);
    return SCPHD_OK;
}

}  // extern "C"
