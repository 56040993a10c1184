// vxsim_config.cpp — RON scene configuration loader (SceneConfig::load,
// src/scene.rs:268-273).
//
// A small recursive-descent reader for the part of RON that scene files use:
// line and (nested) block comments, structs `(field: value, ...)` with an
// optional struct name, tuples `(a, b, c)` for the fixed-size arrays, number
// literals (decimal, hex/octal/binary integers, exponents, `inf`, `NaN`,
// digit separators `_`) and unit enum variants as bare identifiers. Text is
// first read into a value tree, then mapped onto the typed structs with the
// serde rules the reference derives: deny_unknown_fields, every field
// required unless it has a serde default, no field given twice.
#include "vxsim_config.hpp"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <limits>
#include <sstream>
#include <vector>

namespace vxsim {

namespace {

struct Value {
    enum Kind { Number, Ident, Tuple, Struct, Seq, Str } kind = Number;
    std::string text;  // Number: the literal without separators; Ident/Str: the token
    std::string name;  // Struct/Tuple: the optional name before '('
    std::vector<std::pair<std::string, Value>> fields;  // Struct
    std::vector<Value> items;                            // Tuple, Seq
    size_t pos = 0;
};

const char* kind_name(Value::Kind k) {
    switch (k) {
        case Value::Number: return "a number";
        case Value::Ident: return "an identifier";
        case Value::Tuple: return "a tuple";
        case Value::Struct: return "a struct";
        case Value::Seq: return "a sequence";
        case Value::Str: return "a string";
    }
    return "a value";
}

bool ident_start(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_'; }
bool ident_char(char c) { return ident_start(c) || (c >= '0' && c <= '9'); }

class Reader {
public:
    explicit Reader(const std::string& text) : s_(text) {}

    bool document(Value& out) {
        if (!ws()) return false;
        if (!value(out, 0)) return false;
        if (!ws()) return false;
        if (p_ != s_.size()) return fail("trailing characters after the value");
        return true;
    }

    std::string where(size_t pos) const {
        size_t line = 1, col = 1;
        for (size_t k = 0; k < pos && k < s_.size(); ++k) {
            if (s_[k] == '\n') {
                ++line;
                col = 1;
            } else {
                ++col;
            }
        }
        return std::to_string(line) + ":" + std::to_string(col);
    }

    std::string error;

private:
    static constexpr int kMaxDepth = 64;
    const std::string& s_;
    size_t p_ = 0;

    bool fail(const std::string& msg) {
        error = where(p_) + ": " + msg;
        return false;
    }

    // whitespace and comments; block comments nest as in RON
    bool ws() {
        while (p_ < s_.size()) {
            const char c = s_[p_];
            if (c == ' ' || c == '\t' || c == '\n' || c == '\r') {
                ++p_;
            } else if (c == '/' && p_ + 1 < s_.size() && s_[p_ + 1] == '/') {
                while (p_ < s_.size() && s_[p_] != '\n') ++p_;
            } else if (c == '/' && p_ + 1 < s_.size() && s_[p_ + 1] == '*') {
                const size_t start = p_;
                int depth = 0;
                do {
                    if (s_.compare(p_, 2, "/*") == 0) {
                        ++depth;
                        p_ += 2;
                    } else if (s_.compare(p_, 2, "*/") == 0) {
                        --depth;
                        p_ += 2;
                    } else {
                        ++p_;
                    }
                } while (depth > 0 && p_ < s_.size());
                if (depth > 0) {
                    p_ = start;
                    return fail("unterminated block comment");
                }
            } else {
                break;
            }
        }
        return true;
    }

    bool peek(char c) const { return p_ < s_.size() && s_[p_] == c; }

    std::string identifier() {
        const size_t start = p_;
        if (p_ < s_.size() && ident_start(s_[p_])) {
            ++p_;
            while (p_ < s_.size() && ident_char(s_[p_])) ++p_;
        }
        return s_.substr(start, p_ - start);
    }

    bool number(Value& out) {
        out.kind = Value::Number;
        out.pos = p_;
        std::string t;
        if (peek('+') || peek('-')) t += s_[p_++];
        if (p_ < s_.size() && ident_start(s_[p_])) {  // inf / NaN after a sign
            const std::string w = identifier();
            if (w != "inf" && w != "NaN") return fail("expected a number");
            out.text = t + w;
            return true;
        }
        const bool radix = s_.compare(p_, 2, "0x") == 0 || s_.compare(p_, 2, "0o") == 0 || s_.compare(p_, 2, "0b") == 0;
        if (radix) {
            t += s_.substr(p_, 2);
            p_ += 2;
        }
        bool digits = false;
        while (p_ < s_.size()) {
            const char c = s_[p_];
            const bool hex = radix && ((c >= 'a' && c <= 'f') || (c >= 'A' && c <= 'F'));
            if ((c >= '0' && c <= '9') || hex) {
                t += c;
                digits = true;
            } else if (c == '_' && digits) {
                // digit separator
            } else if (!radix && (c == '.' || c == 'e' || c == 'E')) {
                t += c;
                if ((c == 'e' || c == 'E') && p_ + 1 < s_.size() && (s_[p_ + 1] == '+' || s_[p_ + 1] == '-'))
                    t += s_[++p_];
            } else {
                break;
            }
            ++p_;
        }
        if (!digits) return fail("expected a number");
        out.text = t;
        return true;
    }

    bool string(Value& out) {
        out.kind = Value::Str;
        out.pos = p_++;
        std::string t;
        while (p_ < s_.size() && s_[p_] != '"') {
            if (s_[p_] == '\\' && p_ + 1 < s_.size()) ++p_;
            t += s_[p_++];
        }
        if (p_ >= s_.size()) return fail("unterminated string");
        ++p_;
        out.text = t;
        return true;
    }

    // After '(' : a struct when the first entry is `ident:`, else a tuple.
    bool parens(Value& out, int depth) {
        ++p_;
        if (!ws()) return false;
        const size_t save = p_;
        const std::string first = identifier();
        bool is_struct = false;
        if (!first.empty()) {
            if (!ws()) return false;
            is_struct = peek(':');
        }
        p_ = save;
        out.kind = is_struct ? Value::Struct : Value::Tuple;
        while (true) {
            if (!ws()) return false;
            if (peek(')')) {
                ++p_;
                return true;
            }
            if (is_struct) {
                const size_t at = p_;
                const std::string key = identifier();
                if (key.empty()) return fail("expected a field name");
                if (!ws()) return false;
                if (!peek(':')) return fail("expected ':' after field `" + key + "`");
                ++p_;
                if (!ws()) return false;
                Value v;
                if (!value(v, depth + 1)) return false;
                v.pos = at;
                out.fields.emplace_back(key, std::move(v));
            } else {
                Value v;
                if (!value(v, depth + 1)) return false;
                out.items.push_back(std::move(v));
            }
            if (!ws()) return false;
            if (peek(',')) {
                ++p_;
            } else if (!peek(')')) {
                return fail("expected ',' or ')'");
            }
        }
    }

    bool value(Value& out, int depth) {
        if (depth > kMaxDepth) return fail("nesting too deep");
        if (p_ >= s_.size()) return fail("unexpected end of input");
        const size_t at = p_;
        const char c = s_[p_];
        if (c == '(') {
            if (!parens(out, depth)) return false;
            out.pos = at;
            return true;
        }
        if (c == '[') {
            ++p_;
            out.kind = Value::Seq;
            out.pos = at;
            while (true) {
                if (!ws()) return false;
                if (peek(']')) {
                    ++p_;
                    return true;
                }
                Value v;
                if (!value(v, depth + 1)) return false;
                out.items.push_back(std::move(v));
                if (!ws()) return false;
                if (peek(',')) {
                    ++p_;
                } else if (!peek(']')) {
                    return fail("expected ',' or ']'");
                }
            }
        }
        if (c == '"') return string(out);
        if (c == '+' || c == '-' || c == '.' || (c >= '0' && c <= '9')) return number(out);
        if (ident_start(c)) {
            const std::string w = identifier();
            if (w == "inf" || w == "NaN") {
                out.kind = Value::Number;
                out.text = w;
                out.pos = at;
                return true;
            }
            const size_t after = p_;
            if (!ws()) return false;
            if (peek('(')) {  // named struct or tuple
                if (!parens(out, depth)) return false;
                out.name = w;
                out.pos = at;
                return true;
            }
            p_ = after;
            out.kind = Value::Ident;
            out.text = w;
            out.pos = at;
            return true;
        }
        return fail(std::string("unexpected character '") + c + "'");
    }
};

// ---- typed mapping -------------------------------------------------------

struct Mapper {
    const Reader& rd;
    std::string error;

    bool fail(const Value& v, const std::string& msg) {
        error = rd.where(v.pos) + ": " + msg;
        return false;
    }

    bool as_f32(const Value& v, float& out) {
        if (v.kind != Value::Number) return fail(v, std::string("invalid type: ") + kind_name(v.kind) + ", expected f32");
        std::string t = v.text;
        double sign = 1.0;
        if (!t.empty() && (t[0] == '+' || t[0] == '-')) {
            sign = t[0] == '-' ? -1.0 : 1.0;
            t.erase(0, 1);
        }
        if (t == "inf") {
            out = (float)(sign * std::numeric_limits<double>::infinity());
            return true;
        }
        if (t == "NaN") {
            out = std::numeric_limits<float>::quiet_NaN();
            return true;
        }
        if (t.size() > 1 && t[0] == '0' && (t[1] == 'x' || t[1] == 'o' || t[1] == 'b')) {
            uint64_t u = 0;
            if (!radix_u64(v, t, u)) return false;
            out = (float)(sign * (double)u);
            return true;
        }
        // correctly rounded decimal -> f32, as Rust's str::parse::<f32>
        char* end = nullptr;
        errno = 0;
        const float f = std::strtof(t.c_str(), &end);
        if (end == t.c_str() || *end != '\0') return fail(v, "invalid number `" + v.text + "`");
        out = sign < 0 ? -f : f;
        return true;
    }

    bool radix_u64(const Value& v, const std::string& t, uint64_t& out) {
        const int base = t[1] == 'x' ? 16 : (t[1] == 'o' ? 8 : 2);
        uint64_t u = 0;
        for (size_t k = 2; k < t.size(); ++k) {
            const char c = t[k];
            const int d = c <= '9' ? c - '0' : (c | 0x20) - 'a' + 10;
            if (d < 0 || d >= base) return fail(v, "invalid digit in `" + v.text + "`");
            if (u > (std::numeric_limits<uint64_t>::max() - (uint64_t)d) / (uint64_t)base)
                return fail(v, "integer `" + v.text + "` is out of range");
            u = u * (uint64_t)base + (uint64_t)d;
        }
        if (t.size() == 2) return fail(v, "invalid number `" + v.text + "`");
        out = u;
        return true;
    }

    bool as_u64(const Value& v, uint64_t& out, const char* type) {
        if (v.kind != Value::Number)
            return fail(v, std::string("invalid type: ") + kind_name(v.kind) + ", expected " + type);
        std::string t = v.text;
        if (!t.empty() && t[0] == '+') t.erase(0, 1);
        if (!t.empty() && t[0] == '-') return fail(v, std::string("invalid value: `") + v.text + "`, expected " + type);
        if (t.size() > 1 && t[0] == '0' && (t[1] == 'x' || t[1] == 'o' || t[1] == 'b')) return radix_u64(v, t, out);
        if (t.empty() || t.find_first_not_of("0123456789") != std::string::npos)
            return fail(v, std::string("invalid type: floating point `") + v.text + "`, expected " + type);
        uint64_t u = 0;
        for (char c : t) {
            const uint64_t d = (uint64_t)(c - '0');
            if (u > (std::numeric_limits<uint64_t>::max() - d) / 10)
                return fail(v, "integer `" + v.text + "` is out of range");
            u = u * 10 + d;
        }
        out = u;
        return true;
    }

    template <class T, class F>
    bool triple(const Value& v, std::array<T, 3>& out, F&& elem) {
        if (v.kind != Value::Tuple || !v.name.empty())
            return fail(v, std::string("invalid type: ") + kind_name(v.kind) + ", expected a tuple of size 3");
        if (v.items.size() != 3)
            return fail(v, "invalid length " + std::to_string(v.items.size()) + ", expected a tuple of size 3");
        for (int a = 0; a < 3; ++a)
            if (!elem(v.items[a], out[a])) return false;
        return true;
    }
    bool f32x3(const Value& v, std::array<float, 3>& out) {
        return triple(v, out, [this](const Value& e, float& f) { return as_f32(e, f); });
    }
    bool usizex3(const Value& v, std::array<uint64_t, 3>& out) {
        return triple(v, out, [this](const Value& e, uint64_t& u) { return as_u64(e, u, "usize"); });
    }

    using Setter = std::function<bool(const Value&)>;
    struct Field {
        const char* name;
        bool required;
        Setter set;
    };

    // serde's derived struct visitor with deny_unknown_fields
    bool fields(const Value& v, const char* struct_name, const std::vector<Field>& spec) {
        if (v.kind != Value::Struct) {
            if (v.kind == Value::Tuple && v.items.empty()) {  // `()` or `Name()`: every field missing
            } else {
                return fail(v, std::string("invalid type: ") + kind_name(v.kind) + ", expected struct " + struct_name);
            }
        }
        if (!v.name.empty() && v.name != struct_name)
            return fail(v, "expected struct " + std::string(struct_name) + " but found `" + v.name + "`");
        std::vector<bool> seen(spec.size(), false);
        for (const auto& kv : v.fields) {
            size_t k = 0;
            while (k < spec.size() && kv.first != spec[k].name) ++k;
            if (k == spec.size()) {
                std::string expected;
                for (size_t q = 0; q < spec.size(); ++q)
                    expected += std::string(q ? ", `" : "`") + spec[q].name + "`";
                return fail(kv.second, "unknown field `" + kv.first + "`, expected one of " + expected);
            }
            if (seen[k]) return fail(kv.second, "duplicate field `" + kv.first + "`");
            seen[k] = true;
            if (!spec[k].set(kv.second)) return false;
        }
        for (size_t k = 0; k < spec.size(); ++k)
            if (!seen[k] && spec[k].required)
                return fail(v, std::string("missing field `") + spec[k].name + "` in " + struct_name);
        return true;
    }

    bool fracture(const Value& v, FractureSettings& f) {
        auto f32 = [this](float& dst) { return [this, &dst](const Value& x) { return as_f32(x, dst); }; };
        auto u64 = [this](uint64_t& dst, const char* t) {
            return [this, &dst, t](const Value& x) { return as_u64(x, dst, t); };
        };
        return fields(v, "FractureConfig",
                      {{"damage_rate", true, f32(f.damage_rate)},
                       {"energy_release", true, f32(f.energy_release)},
                       {"propagation_delay", true, u64(f.propagation_delay, "u64")},
                       {"fatigue_cycles", true, f32(f.fatigue_cycles)},
                       {"fatigue_exponent", true, f32(f.fatigue_exponent)},
                       {"fatigue_threshold", true, f32(f.fatigue_threshold)},
                       {"plastic_heat_fraction", true, f32(f.plastic_heat_fraction)},
                       {"fragment_min_size", true, u64(f.fragment_min_size, "usize")},
                       {"cluster_interval", true, u64(f.cluster_interval, "u64")},
                       {"friction", true, f32(f.friction)},
                       {"restitution", true, f32(f.restitution)}});
    }

    bool scene(const Value& v, SceneFileConfig& c) {
        auto f32 = [this](float& dst) { return [this, &dst](const Value& x) { return as_f32(x, dst); }; };
        auto usize = [this](uint64_t& dst) { return [this, &dst](const Value& x) { return as_u64(x, dst, "usize"); }; };
        auto vf = [this](std::array<float, 3>& dst) { return [this, &dst](const Value& x) { return f32x3(x, dst); }; };
        auto vu = [this](std::array<uint64_t, 3>& dst) {
            return [this, &dst](const Value& x) { return usizex3(x, dst); };
        };
        auto precond = [this, &c](const Value& x) {
            // CpuPreconditioner, #[serde(rename_all = "snake_case")] (src/scene.rs:14-24)
            if (x.kind != Value::Ident) return fail(x, std::string("invalid type: ") + kind_name(x.kind) + ", expected enum CpuPreconditioner");
            if (x.text != "incomplete_cholesky0" && x.text != "block_jacobi")
                return fail(x, "unknown variant `" + x.text + "`, expected `incomplete_cholesky0` or `block_jacobi`");
            c.cpu_preconditioner = x.text;
            return true;
        };
        auto frac = [this, &c](const Value& x) { return fracture(x, c.fracture); };
        return fields(v, "SceneConfig",
                      {{"dimensions", true, vu(c.dimensions)},
                       {"branch_dimensions", true, vu(c.branch_dimensions)},
                       {"ground_dimensions", true, vu(c.ground_dimensions)},
                       {"tool_dimensions", true, vu(c.tool_dimensions)},
                       {"fibers", true, vf(c.fibers)},
                       {"anisotropy", true, f32(c.anisotropy)},
                       {"gravity", true, vf(c.gravity)},
                       {"fixed_dt", true, f32(c.fixed_dt)},
                       {"substeps", true, usize(c.substeps)},
                       {"iterations", true, usize(c.iterations)},
                       {"cuda_iterations", false, usize(c.cuda_iterations)},
                       {"cpu_preconditioner", false, precond},
                       {"solver_relative_tolerance", true, f32(c.solver_relative_tolerance)},
                       {"corotation_tolerance", true, f32(c.corotation_tolerance)},
                       {"corotation_iterations", true, usize(c.corotation_iterations)},
                       {"fracture", true, frac},
                       {"initial_speed", true, f32(c.initial_speed)},
                       {"tool_start", true, vf(c.tool_start)}});
    }
};

bool in01(float x) { return x >= 0.f && x <= 1.f; }
bool finite3(const std::array<float, 3>& v) {
    return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
}

}  // namespace

// src/fracture.rs:45-60
bool FractureSettings::validate() const {
    return std::isfinite(damage_rate) && damage_rate > 0.f && in01(energy_release) && std::isfinite(fatigue_cycles) &&
           fatigue_cycles > 0.f && std::isfinite(fatigue_exponent) && fatigue_exponent >= 1.f &&
           fatigue_threshold >= 0.f && fatigue_threshold < 1.f && in01(plastic_heat_fraction) &&
           fragment_min_size > 0 && cluster_interval > 0 && std::isfinite(friction) && friction >= 0.f &&
           in01(restitution);
}

// src/scene.rs:275-297
const char* SceneFileConfig::validate() const {
    auto has_zero = [](const std::array<uint64_t, 3>& d) { return d[0] == 0 || d[1] == 0 || d[2] == 0; };
    const float fx = fibers[0], fy = fibers[1], fz = fibers[2];
    const float fiber_len2 = fx * fx + fy * fy + fz * fz;  // Vec3::length_squared in f32
    const bool bad = has_zero(dimensions) || has_zero(ground_dimensions) || tool_dimensions[0] < 2 ||
                     tool_dimensions[1] < 2 || tool_dimensions[2] < 2 || !in01(anisotropy) || !finite3(gravity) ||
                     !finite3(tool_start) || !std::isfinite(initial_speed) || initial_speed < 0.f ||
                     !finite3(fibers) || !std::isfinite(fixed_dt) || fixed_dt <= 0.f || substeps == 0 ||
                     iterations == 0 || cuda_iterations == 0 || corotation_iterations == 0 ||
                     !std::isfinite(solver_relative_tolerance) || solver_relative_tolerance <= 0.f ||
                     !std::isfinite(corotation_tolerance) || corotation_tolerance <= 0.f || !fracture.validate() ||
                     fiber_len2 < 1e-8f;
    return bad ? "Invalid scene parameters" : nullptr;
}

SceneConfig SceneFileConfig::solver_config() const {
    auto u32 = [](uint64_t v) { return (uint32_t)std::min<uint64_t>(v, std::numeric_limits<uint32_t>::max()); };
    SceneConfig c;
    c.gravity = gravity;
    c.fixed_dt = fixed_dt;
    c.substeps = u32(substeps);
    c.iterations = u32(cuda_iterations);  // the device path's cap (src/scene.rs:228-230)
    c.solver_relative_tolerance = solver_relative_tolerance;
    c.corotation_tolerance = corotation_tolerance;
    c.corotation_iterations = u32(corotation_iterations);
    c.fracture = true;
    c.fracture_config.damage_rate = fracture.damage_rate;
    c.fracture_config.energy_release = fracture.energy_release;
    c.fracture_config.fatigue_cycles = fracture.fatigue_cycles;
    c.fracture_config.fatigue_exponent = fracture.fatigue_exponent;
    c.fracture_config.fatigue_threshold = fracture.fatigue_threshold;
    c.fracture_config.plastic_heat_fraction = fracture.plastic_heat_fraction;
    c.contact = true;
    c.restitution = fracture.restitution;
    c.friction = fracture.friction;
    return c;
}

bool parse_scene_config(const std::string& text, SceneFileConfig& out, std::string& error) {
    Reader rd(text);
    Value root;
    if (!rd.document(root)) {
        error = rd.error;
        return false;
    }
    SceneFileConfig c;
    Mapper m{rd, {}};
    if (!m.scene(root, c)) {
        error = m.error;
        return false;
    }
    out = c;
    return true;
}

bool load_scene_config(const std::string& path, SceneFileConfig& out, std::string& error) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        error = path + ": cannot open";
        return false;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    SceneFileConfig c;
    if (!parse_scene_config(ss.str(), c, error)) return false;
    if (const char* why = c.validate()) {
        error = why;
        return false;
    }
    out = c;
    return true;
}

}  // namespace vxsim
