// Settings of the B200 engine: the reference's full key set (src/settings.zig:38-178), JSON in
// and out (src/settings.zig:198-223). The key table keeps the reference's names, order, types
// and defaults; it is the interface the reference's Python layer validates keyword arguments
// against (python/zcmir/api.py:65-84), so it has to match key for key.
#include "settings.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

namespace zc {
namespace {

const char* const kMetric[] = {"smi", "smi_edge", "e4", "lmax", "ncc", nullptr};
const char* const kDetector[] = {"pos_gift", "gls_mift", nullptr};
const char* const kMatchMethod[] = {"lofsc", "prosac", "magsac", nullptr};
const char* const kSearchMode[] = {"sweep", "cloud", nullptr};
const char* const kSmiFeatures[] = {"laplacian", "three", "cubic", nullptr};
const char* const kGroup[] = {"affine", "homography", nullptr};
const char* const kSizes[] = {"ladder", "compact", nullptr};

const KeyDef kKeys[] = {
    {"metric", Kind::Enum, kMetric, 0, "smi"},
    {"smi_features", Kind::Enum, kSmiFeatures, 0, "laplacian"},
    {"exact", Kind::Bool, nullptr, 1, nullptr},
    {"calibrated", Kind::Bool, nullptr, 1, nullptr},
    {"symmetric", Kind::Bool, nullptr, 1, nullptr},
    {"group", Kind::Enum, kGroup, 0, "homography"},
    {"map_res", Kind::U32, nullptr, 0, nullptr},
    {"min_overlap", Kind::F64, nullptr, 0.05, nullptr},
    {"rs_smin", Kind::F64, nullptr, 0.2, nullptr},
    {"rs_smax", Kind::F64, nullptr, 5.0, nullptr},
    {"ffd", Kind::Bool, nullptr, 0, nullptr},
    {"ffd_grid", Kind::U32, nullptr, 4, nullptr},
    {"ffd_source", Kind::Bool, nullptr, 0, nullptr},
    {"ffd_stiffness", Kind::F64, nullptr, 0.15, nullptr},
    {"hop", Kind::Bool, nullptr, 1, nullptr},
    {"hop_fm", Kind::Bool, nullptr, 0, nullptr},
    {"g_a0", Kind::F64, nullptr, 0.08, nullptr},
    {"g_decay", Kind::F64, nullptr, 0.5, nullptr},
    {"g_steps", Kind::U32, nullptr, 7, nullptr},
    {"g_iters", Kind::U32, nullptr, 100, nullptr},
    {"clahe", Kind::Bool, nullptr, 1, nullptr},
    {"clahe_grid", Kind::U32, nullptr, 4, nullptr},
    {"clahe_bins", Kind::U32, nullptr, 64, nullptr},
    {"band", Kind::Bool, nullptr, 0, nullptr},
    {"bp_fine", Kind::F64, nullptr, 1.0, nullptr},
    {"bp_coarse", Kind::F64, nullptr, 6.0, nullptr},
    {"invert", Kind::Bool, nullptr, 0, nullptr},
    {"half", Kind::Bool, nullptr, 1, nullptr},
    {"fft_sizes", Kind::Enum, kSizes, 0, "ladder"},
    {"detector", Kind::Enum, kDetector, 0, "pos_gift"},
    {"n_octaves", Kind::U32, nullptr, 3, nullptr},
    {"max_points", Kind::U32, nullptr, 2000, nullptr},
    {"min_contrast", Kind::F64, nullptr, 0.01, nullptr},
    {"tau", Kind::F64, nullptr, 0.8, nullptr},
    {"radius", Kind::F64, nullptr, 36.0, nullptr},
    {"nt", Kind::F64, nullptr, 0.0, nullptr},
    {"auto_nt", Kind::Bool, nullptr, 1, nullptr},
    {"second_ori", Kind::Bool, nullptr, 1, nullptr},
    {"inlier_px", Kind::F64, nullptr, 10.0, nullptr},
    {"scale_lo", Kind::F64, nullptr, 0.2, nullptr},
    {"scale_hi", Kind::F64, nullptr, 5.0, nullptr},
    {"max_aniso", Kind::F64, nullptr, 5.0, nullptr},
    {"max_persp", Kind::F64, nullptr, 3.0, nullptr},
    {"n_trials", Kind::U32, nullptr, 100000, nullptr},
    {"seed", Kind::U32, nullptr, 12345, nullptr},
    {"n_sigma", Kind::U32, nullptr, 4, nullptr},
    {"n_angle", Kind::U32, nullptr, 6, nullptr},
    {"n_r", Kind::U32, nullptr, 3, nullptr},
    {"match_method", Kind::Enum, kMatchMethod, 0, "lofsc"},
    {"per_octave", Kind::Bool, nullptr, 1, nullptr},
    {"mutual", Kind::Bool, nullptr, 0, nullptr},
    {"pg_n_octaves", Kind::U32, nullptr, 3, nullptr},
    {"pg_max_points", Kind::U32, nullptr, 5000, nullptr},
    {"pg_min_contrast", Kind::F64, nullptr, 0.01, nullptr},
    {"pg_p1", Kind::F64, nullptr, 10.0, nullptr},
    {"pg_search", Kind::Bool, nullptr, 1, nullptr},
    {"pg_corners", Kind::Bool, nullptr, 1, nullptr},
    {"pg_desc_pow", Kind::F64, nullptr, 1.5, nullptr},
    {"pg_n_orient", Kind::U32, nullptr, 6, nullptr},
    {"pg_n_rings", Kind::U32, nullptr, 3, nullptr},
    {"pg_n_scales", Kind::U32, nullptr, 4, nullptr},
    {"pg_min_wl", Kind::F64, nullptr, 3.0, nullptr},
    {"pg_mult", Kind::F64, nullptr, 1.6, nullptr},
    {"pg_sigma_onf", Kind::F64, nullptr, 0.75, nullptr},
    {"pg_pc_k", Kind::F64, nullptr, 1.0, nullptr},
    {"pg_cutoff", Kind::F64, nullptr, 0.5, nullptr},
    {"pg_pc_g", Kind::F64, nullptr, 3.0, nullptr},
    {"pg_gsig", Kind::F64, nullptr, 3.0, nullptr},
    {"pg_pos_p1", Kind::F64, nullptr, 20.0, nullptr},
    {"pg_pos_k", Kind::U32, nullptr, 20, nullptr},
    {"pg_ratio", Kind::F64, nullptr, 0.6, nullptr},
    {"pg_pos", Kind::Bool, nullptr, 1, nullptr},
    {"pg_pos_search_px", Kind::F64, nullptr, 10.0, nullptr},
    {"pg_pos_px", Kind::F64, nullptr, 3.0, nullptr},
    {"pg_released", Kind::Bool, nullptr, 0, nullptr},
    {"search_mode", Kind::Enum, kSearchMode, 0, "sweep"},
    {"sw_grid", Kind::U32, nullptr, 128, nullptr},
    {"sw_nth", Kind::U32, nullptr, 90, nullptr},
    {"sw_rot", Kind::F64, nullptr, 180.0, nullptr},
    {"sw_rot_range", Kind::Bool, nullptr, 0, nullptr},
    {"sw_rot_lo", Kind::F64, nullptr, -180.0, nullptr},
    {"sw_rot_hi", Kind::F64, nullptr, 180.0, nullptr},
    {"sw_shear", Kind::Bool, nullptr, 0, nullptr},
    {"sw_shear_max", Kind::F64, nullptr, 0.1, nullptr},
    {"sw_nshear", Kind::U32, nullptr, 3, nullptr},
    {"sw_aniso", Kind::Bool, nullptr, 0, nullptr},
    {"sw_aniso_max", Kind::F64, nullptr, 0.1, nullptr},
    {"sw_naniso", Kind::U32, nullptr, 3, nullptr},
    {"sw_ns", Kind::U32, nullptr, 20, nullptr},
    {"sw_smin", Kind::F64, nullptr, 0.5, nullptr},
    {"sw_smax", Kind::F64, nullptr, 2.0, nullptr},
    {"sw_k", Kind::U32, nullptr, 32, nullptr},
    {"sw_fin", Kind::U32, nullptr, 4, nullptr},
    {"sw_rel", Kind::Bool, nullptr, 0, nullptr},
    {"hho_auto", Kind::Bool, nullptr, 1, nullptr},
    {"hho_n", Kind::U32, nullptr, 100, nullptr},
    {"hho_t", Kind::U32, nullptr, 20, nullptr},
    {"hho_sg", Kind::F64, nullptr, 0.01, nullptr},
    {"hho_sh", Kind::F64, nullptr, 0.01, nullptr},
    {"hho_p", Kind::F64, nullptr, 0.0001, nullptr},
    {"hho_tx", Kind::F64, nullptr, 0.01, nullptr},
    {"hho_th", Kind::F64, nullptr, 0.01, nullptr},
    {"hho_phi", Kind::F64, nullptr, 0.01, nullptr},
    {"hho_seed", Kind::U32, nullptr, 1, nullptr},
    {"hho_rel", Kind::Bool, nullptr, 1, nullptr},
};

constexpr int kNumKeys = sizeof(kKeys) / sizeof(kKeys[0]);

// ── a small JSON reader: one flat object of scalars (nested values are rejected) ──

struct JVal {
    enum T { Null, Bool, Num, Str } t = Null;
    bool b = false;
    double num = 0;
    bool integral = false;
    std::string s;
};

struct Parser {
    const char* p;
    const char* end;
    std::string err;

    void ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
    }
    bool fail(const char* m) {
        if (err.empty()) err = m;
        return false;
    }
    bool str(std::string& out) {
        if (p >= end || *p != '"') return fail("expected a string");
        ++p;
        out.clear();
        while (p < end && *p != '"') {
            char c = *p++;
            if (c == '\\') {
                if (p >= end) return fail("bad escape");
                char e = *p++;
                switch (e) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        if (end - p < 4) return fail("bad escape");
                        unsigned cp = (unsigned)strtoul(std::string(p, 4).c_str(), nullptr, 16);
                        p += 4;
                        if (cp < 0x80) out += (char)cp;
                        else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
                        else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
                        break;
                    }
                    default: return fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        if (p >= end) return fail("unterminated string");
        ++p;
        return true;
    }
    bool value(JVal& v) {
        ws();
        if (p >= end) return fail("expected a value");
        if (*p == '"') {
            v.t = JVal::Str;
            return str(v.s);
        }
        if (end - p >= 4 && !strncmp(p, "true", 4)) { v.t = JVal::Bool; v.b = true; p += 4; return true; }
        if (end - p >= 5 && !strncmp(p, "false", 5)) { v.t = JVal::Bool; v.b = false; p += 5; return true; }
        if (end - p >= 4 && !strncmp(p, "null", 4)) { v.t = JVal::Null; p += 4; return true; }
        if (*p == '{' || *p == '[') return fail("nested values are not settings");
        const char* s = p;
        if (p < end && (*p == '-' || *p == '+')) ++p;
        bool frac = false;
        while (p < end && (isdigit((unsigned char)*p) || *p == '.' || *p == 'e' || *p == 'E' || *p == '-' || *p == '+')) {
            if (*p == '.' || *p == 'e' || *p == 'E') frac = true;
            ++p;
        }
        if (p == s) return fail("expected a value");
        std::string t(s, p);
        char* q = nullptr;
        v.num = strtod(t.c_str(), &q);
        if (!q || *q) return fail("bad number");
        v.t = JVal::Num;
        v.integral = !frac || (std::isfinite(v.num) && std::floor(v.num) == v.num);
        return true;
    }
};

std::string fmt_num(double v) {
    char buf[64];
    for (int prec = 15; prec <= 17; ++prec) {
        snprintf(buf, sizeof buf, "%.*g", prec, v);
        if (strtod(buf, nullptr) == v) break;
    }
    std::string s(buf);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";  // keep floats floats
    return s;
}

}  // namespace

int Settings::count() { return kNumKeys; }
const KeyDef& Settings::def(int i) { return kKeys[i]; }

int Settings::index_of(const std::string& key) {
    for (int i = 0; i < kNumKeys; ++i)
        if (key == kKeys[i].name) return i;
    return -1;
}

Settings::Settings() : num_(kNumKeys), str_(kNumKeys) {
    for (int i = 0; i < kNumKeys; ++i) {
        num_[i] = kKeys[i].dnum;
        if (kKeys[i].dstr) str_[i] = kKeys[i].dstr;
    }
}

bool Settings::apply(const char* json, size_t len, std::string& err) {
    Parser ps{json, json + len, {}};
    std::vector<double> num = num_;
    std::vector<std::string> str = str_;
    ps.ws();
    if (ps.p >= ps.end || *ps.p != '{') {
        err = "configure: ExpectedObject";
        return false;
    }
    ++ps.p;
    ps.ws();
    if (ps.p < ps.end && *ps.p == '}') {
        ++ps.p;
    } else {
        while (true) {
            ps.ws();
            std::string key;
            if (!ps.str(key)) { err = "configure: " + ps.err; return false; }
            ps.ws();
            if (ps.p >= ps.end || *ps.p != ':') { err = "configure: expected ':'"; return false; }
            ++ps.p;
            JVal v;
            if (!ps.value(v)) { err = "configure: " + ps.err; return false; }
            const int i = index_of(key);
            if (i < 0) { err = "configure: UnknownSetting (" + key + ")"; return false; }
            const KeyDef& d = kKeys[i];
            switch (d.kind) {
                case Kind::Bool:
                    if (v.t != JVal::Bool) { err = "configure: UnexpectedToken (" + key + ": expected a bool)"; return false; }
                    num[i] = v.b ? 1 : 0;
                    break;
                case Kind::U32:
                    if (v.t != JVal::Num || !v.integral || v.num < 0 || v.num > 4294967295.0) {
                        err = "configure: InvalidNumber (" + key + ": expected an unsigned 32-bit integer)";
                        return false;
                    }
                    num[i] = v.num;
                    break;
                case Kind::F64:
                    if (v.t != JVal::Num) { err = "configure: UnexpectedToken (" + key + ": expected a number)"; return false; }
                    num[i] = v.num;
                    break;
                case Kind::Enum: {
                    bool ok = false;
                    if (v.t == JVal::Str)
                        for (const char* const* e = d.values; *e; ++e) ok = ok || v.s == *e;
                    if (!ok) { err = "configure: InvalidEnumTag (" + key + ")"; return false; }
                    str[i] = v.s;
                    break;
                }
            }
            ps.ws();
            if (ps.p < ps.end && *ps.p == ',') { ++ps.p; continue; }
            if (ps.p < ps.end && *ps.p == '}') { ++ps.p; break; }
            err = "configure: expected ',' or '}'";
            return false;
        }
    }
    ps.ws();
    if (ps.p != ps.end) { err = "configure: trailing characters"; return false; }
    num_.swap(num);
    str_.swap(str);
    return true;
}

std::string Settings::to_json() const {
    std::string o = "{";
    for (int i = 0; i < kNumKeys; ++i) {
        if (i) o += ",";
        o += "\"";
        o += kKeys[i].name;
        o += "\":";
        switch (kKeys[i].kind) {
            case Kind::Bool: o += num_[i] != 0 ? "true" : "false"; break;
            case Kind::U32: { char b[32]; snprintf(b, sizeof b, "%u", (unsigned)num_[i]); o += b; break; }
            case Kind::F64: o += fmt_num(num_[i]); break;
            case Kind::Enum: o += "\"" + str_[i] + "\""; break;
        }
    }
    return o + "}";
}

static int must(const char* key) {
    const int i = Settings::index_of(key);
    if (i < 0) throw std::logic_error(std::string("no setting ") + key);
    return i;
}

bool Settings::b(const char* key) const { return num_[must(key)] != 0; }
double Settings::f(const char* key) const { return num_[must(key)]; }
unsigned Settings::u(const char* key) const { return (unsigned)num_[must(key)]; }
const std::string& Settings::e(const char* key) const { return str_[must(key)]; }

}  // namespace zc
