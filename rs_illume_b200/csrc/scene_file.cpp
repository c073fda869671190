// pbrt-v3 scene files -> shapes, materials, camera and render settings.
//
// The reference parses these files into a syntax tree (parse_to_ast,
// core/parser/mod.rs:19-34, with the grammar of core/parser/parsers/ and the
// tree of core/parser/ast.rs) and has a ParamSet for typed parameter lookup
// (core/paramset.rs:303-511), but its parse() constructs nothing from the
// tree (core/parser/mod.rs:36-46).  This file tokenises the text, reads each
// directive's arguments with one grammar table (Reader::read_directive), runs
// the directive against pbrt's graphics state and keeps what the ray-query
// and path-tracing library can represent; directive semantics and parameter
// defaults follow pbrt-v3 (api.cpp and the shape / material / camera
// factories).  ilm_scene_syntax returns the directive tree that the same
// reader produces, without running it, for comparison with the reference's
// parser tests.
//
// Transforms are kept in double precision as (matrix, inverse) pairs and
// rounded to float when a shape takes them.  Normals go through the inverse
// transpose (core/transform.rs:337-344 multiplies by the matrix's transpose,
// which is right only for rotations).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "builder.h"
#include "illume_gpu.h"

namespace {

constexpr double kPiD = 3.14159265358979323846;

// ----------------------------------------------------------------- transforms
struct Mat4 {
    double m[4][4];
};

Mat4 identity4() {
    Mat4 r{};
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0;
    return r;
}

Mat4 mul4(const Mat4& a, const Mat4& b) {
    Mat4 r{};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a.m[i][k] * b.m[k][j];
            r.m[i][j] = s;
        }
    return r;
}

Mat4 transpose4(const Mat4& a) {
    Mat4 r{};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) r.m[i][j] = a.m[j][i];
    return r;
}

// Gauss-Jordan with partial pivoting; false for a singular matrix.
bool invert4(const Mat4& a, Mat4* out) {
    double w[4][8];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 8; ++j) w[i][j] = j < 4 ? a.m[i][j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(w[r][c]) > std::fabs(w[p][c])) p = r;
        if (w[p][c] == 0.0 || !std::isfinite(w[p][c])) return false;
        if (p != c)
            for (int j = 0; j < 8; ++j) std::swap(w[p][j], w[c][j]);
        double inv = 1.0 / w[c][c];
        for (int j = 0; j < 8; ++j) w[c][j] *= inv;
        for (int r = 0; r < 4; ++r) {
            if (r == c || w[r][c] == 0.0) continue;
            double f = w[r][c];
            for (int j = 0; j < 8; ++j) w[r][j] -= f * w[c][j];
        }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out->m[i][j] = w[i][j + 4];
    return true;
}

struct Xform {
    Mat4 m = identity4(), inv = identity4();
};

Xform compose(const Xform& a, const Xform& b) { return Xform{mul4(a.m, b.m), mul4(b.inv, a.inv)}; }

double det3(const Mat4& a) {
    return a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
           a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
           a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
}

// Transform::translate / scale / rotate / look_at (core/transform.rs:63-209).
Xform translate(double x, double y, double z) {
    Xform t;
    t.m.m[0][3] = x; t.m.m[1][3] = y; t.m.m[2][3] = z;
    t.inv.m[0][3] = -x; t.inv.m[1][3] = -y; t.inv.m[2][3] = -z;
    return t;
}

Xform scale(double x, double y, double z) {
    Xform t;
    t.m.m[0][0] = x; t.m.m[1][1] = y; t.m.m[2][2] = z;
    t.inv.m[0][0] = 1.0 / x; t.inv.m[1][1] = 1.0 / y; t.inv.m[2][2] = 1.0 / z;
    return t;
}

Xform rotate(double deg, double ax, double ay, double az) {
    double len = std::sqrt(ax * ax + ay * ay + az * az);
    ax /= len; ay /= len; az /= len;
    double th = deg * kPiD / 180.0, s = std::sin(th), c = std::cos(th);
    Xform t;
    double (*m)[4] = t.m.m;
    m[0][0] = ax * ax + (1 - ax * ax) * c;
    m[0][1] = ax * ay * (1 - c) - az * s;
    m[0][2] = ax * az * (1 - c) + ay * s;
    m[1][0] = ax * ay * (1 - c) + az * s;
    m[1][1] = ay * ay + (1 - ay * ay) * c;
    m[1][2] = ay * az * (1 - c) - ax * s;
    m[2][0] = ax * az * (1 - c) - ay * s;
    m[2][1] = ay * az * (1 - c) + ax * s;
    m[2][2] = az * az + (1 - az * az) * c;
    t.inv = transpose4(t.m);
    return t;
}

// World-to-camera of a camera at `pos` looking at `look` with `up`; false
// when up is parallel to the viewing direction.
bool look_at(const double pos[3], const double look[3], const double up[3], Xform* out) {
    double dir[3] = {look[0] - pos[0], look[1] - pos[1], look[2] - pos[2]};
    double dl = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    double ul = std::sqrt(up[0] * up[0] + up[1] * up[1] + up[2] * up[2]);
    if (!(dl > 0.0) || !(ul > 0.0)) return false;
    for (double& v : dir) v /= dl;
    double u[3] = {up[0] / ul, up[1] / ul, up[2] / ul};
    double right[3] = {u[1] * dir[2] - u[2] * dir[1], u[2] * dir[0] - u[0] * dir[2], u[0] * dir[1] - u[1] * dir[0]};
    double rl = std::sqrt(right[0] * right[0] + right[1] * right[1] + right[2] * right[2]);
    if (!(rl > 1e-12)) return false;
    for (double& v : right) v /= rl;
    double nu[3] = {dir[1] * right[2] - dir[2] * right[1], dir[2] * right[0] - dir[0] * right[2],
                    dir[0] * right[1] - dir[1] * right[0]};
    Mat4 c2w = identity4();
    for (int i = 0; i < 3; ++i) {
        c2w.m[i][0] = right[i];
        c2w.m[i][1] = nu[i];
        c2w.m[i][2] = dir[i];
        c2w.m[i][3] = pos[i];
    }
    Mat4 w2c;
    if (!invert4(c2w, &w2c)) return false;
    *out = Xform{w2c, c2w};
    return true;
}

// ------------------------------------------------------------------ tokens
struct Token {
    std::string text;
    bool quoted = false;
    int line = 0;
    int file = 0;     // index into Parser::files_
};

[[noreturn]] void fail_at(const std::string& file, int line, const std::string& msg) {
    throw std::runtime_error(file + ":" + std::to_string(line) + ": " + msg);
}

// Whitespace and '#' comments separate tokens; a comment runs to the end of
// its line.  `comments`, when given, receives each comment's text after '#'.
void tokenize(const std::string& src, int file, const std::string& fname, std::vector<Token>& out,
              std::vector<std::string>* comments = nullptr) {
    int line = 1;
    size_t i = 0, n = src.size();
    while (i < n) {
        char c = src[i];
        if (c == '\n') { ++line; ++i; continue; }
        if (std::isspace((unsigned char)c)) { ++i; continue; }
        if (c == '#') {
            size_t j = i + 1;
            while (j < n && src[j] != '\n') ++j;
            if (comments) comments->push_back(src.substr(i + 1, j - i - 1));
            i = j;
            continue;
        }
        Token t;
        t.line = line;
        t.file = file;
        if (c == '[' || c == ']') {
            t.text = std::string(1, c);
            ++i;
        } else if (c == '"') {
            size_t j = i + 1;
            while (j < n && src[j] != '"') {
                if (src[j] == '\n') fail_at(fname, line, "unterminated string");
                ++j;
            }
            if (j >= n) fail_at(fname, line, "unterminated string");
            t.text = src.substr(i + 1, j - i - 1);
            t.quoted = true;
            i = j + 1;
        } else {
            size_t j = i;
            while (j < n && !std::isspace((unsigned char)src[j]) && src[j] != '[' && src[j] != ']' && src[j] != '"' &&
                   src[j] != '#')
                ++j;
            t.text = src.substr(i, j - i);
            i = j;
        }
        out.push_back(std::move(t));
    }
}

// ------------------------------------------------------------------ params
// One "type name" [values] entry of a parameter list (ParamSetItem,
// core/paramset.rs:11-40).
struct Param {
    std::string type, name;
    std::vector<double> num;
    std::vector<std::string> str;
    bool is_string = false;
    int line = 0;
    mutable bool used = false;
};

struct Params {
    std::vector<Param> items;
    std::string file;

    const Param* find(const char* name, std::initializer_list<const char*> types) const {
        for (const Param& p : items) {
            if (p.name != name) continue;
            for (const char* t : types)
                if (p.type == t) { p.used = true; return &p; }
        }
        return nullptr;
    }
    const Param* need_num(const char* name, std::initializer_list<const char*> types, size_t multiple) const {
        const Param* p = find(name, types);
        if (!p) return nullptr;
        if (p->is_string) fail_at(file, p->line, std::string("parameter \"") + name + "\" needs numbers");
        if (p->num.empty() || p->num.size() % multiple)
            fail_at(file, p->line, std::string("parameter \"") + name + "\" needs a multiple of " +
                                       std::to_string(multiple) + " values");
        return p;
    }
    // ParamSet::find_one_float / find_one_int (paramset.rs:303-322)
    double one_float(const char* name, double def) const {
        const Param* p = need_num(name, {"float"}, 1);
        return p ? p->num[0] : def;
    }
    long one_int(const char* name, long def) const {
        const Param* p = need_num(name, {"integer"}, 1);
        return p ? (long)p->num[0] : def;
    }
    std::string one_string(const char* name, const std::string& def) const {
        const Param* p = find(name, {"string", "bool"});
        if (!p) return def;
        if (!p->is_string || p->str.empty()) fail_at(file, p->line, std::string("parameter \"") + name + "\" needs a string");
        return p->str[0];
    }
    bool one_bool(const char* name, bool def) const {
        const Param* p = find(name, {"bool"});
        if (!p) return def;
        std::string v = p->is_string && !p->str.empty() ? p->str[0] : "";
        if (v == "true") return true;
        if (v == "false") return false;
        fail_at(file, p->line, std::string("parameter \"") + name + "\" needs \"true\" or \"false\"");
    }
    bool point3(const char* name, double out[3]) const {
        const Param* p = need_num(name, {"point", "point3"}, 3);
        if (!p) return false;
        for (int k = 0; k < 3; ++k) out[k] = p->num[k];
        return true;
    }
    // An RGB spectrum parameter ("rgb" / "color"); other spectrum kinds are
    // reported and give the default.
    bool rgb(const char* name, double out[3], std::vector<std::string>& warn) const {
        if (const Param* p = need_num(name, {"rgb", "color"}, 3)) {
            for (int k = 0; k < 3; ++k) out[k] = p->num[k];
            return true;
        }
        if (const Param* p = find(name, {"spectrum", "blackbody", "xyz"})) {
            warn.push_back(file + ":" + std::to_string(p->line) + ": \"" + p->type + " " + name +
                           "\" is not supported; using the default");
            return false;
        }
        if (const Param* p = find(name, {"texture"})) {
            warn.push_back(file + ":" + std::to_string(p->line) + ": texture \"" + name +
                           "\" is not supported; using the default");
            return false;
        }
        return false;
    }
    void report_unused(const std::string& where, std::vector<std::string>& warn) const {
        for (const Param& p : items)
            if (!p.used)
                warn.push_back(file + ":" + std::to_string(p.line) + ": parameter \"" + p.type + " " + p.name +
                               "\" unused by " + where);
    }
};

// ------------------------------------------------------------------ output
struct MeshOut {
    std::vector<float> xyz, n, s, uv;
    std::vector<uint32_t> idx;
    uint32_t material = 0;
};

struct MaterialKey {
    float albedo[3], emission[3];
    bool operator<(const MaterialKey& o) const {
        return std::lexicographical_compare(albedo, albedo + 3, o.albedo, o.albedo + 3) ||
               (std::equal(albedo, albedo + 3, o.albedo) &&
                std::lexicographical_compare(emission, emission + 3, o.emission, o.emission + 3));
    }
};

}  // namespace

struct ilm_scene_file {
    std::vector<MeshOut> meshes;
    std::vector<ilm_sphere_desc> quadrics;
    std::vector<uint32_t> quadric_material;
    std::vector<ilm_curve_desc> curves;
    std::vector<uint32_t> curve_material;
    std::vector<MaterialKey> materials;
    ilm_scene_file_info info{};
    std::string warnings;
};

namespace {

struct ShapeRecord {     // a shape inside ObjectBegin / ObjectEnd
    std::string type;
    Params params;
    Xform ctm;
    bool reverse;
    uint32_t material;
    int line;
};

struct GState {
    Xform ctm;
    bool reverse = false;
    double kd[3] = {0.5, 0.5, 0.5};
    bool emits = false;
    double le[3] = {0, 0, 0};
};

// ------------------------------------------------------------------ reader
// A directive as read from the token stream: its name token, the arguments
// its grammar fixes (numbers, quoted strings, or one bare word) and its
// parameter list.
struct Directive {
    Token tok;
    std::vector<double> num;
    std::vector<std::string> str;
    Params params;
};

// Argument grammar of one directive: `numbers` numbers (bracketed or not),
// `quoted` quoted strings and up to `more_quoted` further ones, or one bare
// `word`; `params` when a parameter list follows.  The directives and their
// arguments are those of core/parser/parsers/directives.rs and transforms.rs
// (pbrt-v3's file format).
struct Grammar {
    int numbers = 0, quoted = 0, more_quoted = 0;
    bool word = false, params = false;
};

const std::map<std::string, Grammar>& grammar() {
    static const std::map<std::string, Grammar> g = [] {
        std::map<std::string, Grammar> m;
        auto nums = [](int k) { Grammar x; x.numbers = k; return x; };
        auto names = [](int k, bool params) { Grammar x; x.quoted = k; x.params = params; return x; };
        for (const char* d : {"Identity", "ReverseOrientation", "WorldBegin", "WorldEnd", "AttributeBegin",
                              "AttributeEnd", "TransformBegin", "TransformEnd", "ObjectEnd"})
            m[d] = Grammar();
        m["Translate"] = nums(3);
        m["Scale"] = nums(3);
        m["Rotate"] = nums(4);
        m["LookAt"] = nums(9);
        m["Transform"] = nums(16);
        m["ConcatTransform"] = nums(16);
        m["TransformTimes"] = nums(2);
        Grammar w;
        w.word = true;
        m["ActiveTransform"] = w;
        for (const char* d : {"CoordinateSystem", "CoordSysTransform", "ObjectBegin", "ObjectInstance",
                              "NamedMaterial", "Include"})
            m[d] = names(1, false);
        for (const char* d : {"Shape", "Material", "MakeNamedMaterial", "AreaLightSource", "LightSource", "Camera",
                              "Film", "Sampler", "Integrator", "PixelFilter", "Accelerator", "MakeNamedMedium"})
            m[d] = names(1, true);
        m["Texture"] = names(3, true);
        Grammar mi = names(1, false);
        mi.more_quoted = 1;
        m["MediumInterface"] = mi;
        return m;
    }();
    return g;
}

// Token-level reading shared by the loader and the syntax dump.
class Reader {
public:
    // The next directive and its arguments, by the grammar table.
    Directive read_directive(const std::vector<Token>& toks, size_t& i) const {
        Directive D;
        D.tok = toks[i++];
        const Token& d = D.tok;
        if (d.quoted || d.text == "[" || d.text == "]") fail(d, "expected a directive, found \"" + d.text + "\"");
        auto it = grammar().find(d.text);
        if (it == grammar().end()) fail(d, "unknown directive \"" + d.text + "\"");
        const Grammar& g = it->second;
        if (g.numbers) D.num = numbers(toks, i, d, (size_t)g.numbers);
        for (int k = 0; k < g.quoted; ++k) D.str.push_back(quoted(toks, i, d));
        for (int k = 0; k < g.more_quoted && i < toks.size() && toks[i].quoted; ++k) D.str.push_back(toks[i++].text);
        if (g.word) {
            const Token& w = next(toks, i, d);
            if (w.quoted || (w.text != "StartTime" && w.text != "EndTime" && w.text != "All"))
                fail(w, d.text + " takes StartTime, EndTime or All");
            D.str.push_back(w.text);
        }
        if (g.params) D.params = params(toks, i);
        return D;
    }

protected:
    std::vector<std::string> files_;

    const std::string& fname(const Token& t) const { return files_[t.file]; }

    [[noreturn]] void fail(const Token& t, const std::string& msg) const { fail_at(fname(t), t.line, msg); }

    const Token& next(const std::vector<Token>& toks, size_t& i, const Token& ctx) const {
        if (i >= toks.size()) fail(ctx, "unexpected end of input after " + ctx.text);
        return toks[i++];
    }

    double number(const Token& t) const {
        if (t.quoted || t.text == "[" || t.text == "]") fail(t, "expected a number, found \"" + t.text + "\"");
        char* end = nullptr;
        errno = 0;
        double v = std::strtod(t.text.c_str(), &end);
        if (end != t.text.c_str() + t.text.size() || errno == ERANGE || !std::isfinite(v))
            fail(t, "expected a number, found \"" + t.text + "\"");
        return v;
    }

    std::vector<double> numbers(const std::vector<Token>& toks, size_t& i, const Token& dir, size_t count) const {
        std::vector<double> v;
        bool bracket = i < toks.size() && !toks[i].quoted && toks[i].text == "[";
        if (bracket) ++i;
        while (v.size() < count) v.push_back(number(next(toks, i, dir)));
        if (bracket) {
            const Token& t = next(toks, i, dir);
            if (t.quoted || t.text != "]") fail(t, dir.text + " takes " + std::to_string(count) + " numbers");
        }
        return v;
    }

    std::string quoted(const std::vector<Token>& toks, size_t& i, const Token& dir) const {
        const Token& t = next(toks, i, dir);
        if (!t.quoted) fail(t, dir.text + " expects a quoted string, found " + t.text);
        return t.text;
    }

    // "type name" value | "type name" [ values ]
    Params params(const std::vector<Token>& toks, size_t& i) const {
        Params ps;
        while (i < toks.size() && toks[i].quoted) {
            const Token& decl = toks[i++];
            std::istringstream ds(decl.text);
            Param p;
            ds >> p.type >> p.name;
            std::string extra;
            if (p.type.empty() || p.name.empty() || (ds >> extra))
                fail(decl, "malformed parameter declaration \"" + decl.text + "\"");
            if (p.type == "point3") p.type = "point";
            if (p.type == "vector3") p.type = "vector";
            if (p.type == "normal3") p.type = "normal";
            static const std::set<std::string> known = {"integer", "float", "point2", "vector2", "point", "vector",
                                                        "normal", "rgb", "color", "xyz", "spectrum", "blackbody",
                                                        "bool", "string", "texture"};
            if (!known.count(p.type)) fail(decl, "unknown parameter type \"" + p.type + "\"");
            p.is_string = p.type == "string" || p.type == "bool" || p.type == "texture" ||
                          (p.type == "spectrum" && i < toks.size() && (toks[i].quoted ||
                           (toks[i].text == "[" && i + 1 < toks.size() && toks[i + 1].quoted)));
            p.line = decl.line;
            const Token& first = next(toks, i, decl);
            // integers are -?digits and booleans "true" or "false", as the
            // reference's grammar reads them (parse_int, values.rs;
            // parse_boolean_parameter, parameters.rs)
            auto take = [&](const Token& t) {
                if (p.is_string) {
                    if (!t.quoted) fail(t, "parameter \"" + p.name + "\" takes quoted strings");
                    if (p.type == "bool" && t.text != "true" && t.text != "false")
                        fail(t, "parameter \"" + p.name + "\" takes \"true\" or \"false\"");
                    p.str.push_back(t.text);
                } else {
                    if (p.type == "integer") {
                        size_t k = !t.quoted && !t.text.empty() && t.text[0] == '-' ? 1 : 0;
                        bool digits = !t.quoted && k < t.text.size();
                        for (size_t j = k; j < t.text.size(); ++j) digits = digits && std::isdigit((unsigned char)t.text[j]);
                        if (!digits) fail(t, "parameter \"" + p.name + "\" takes integers, found \"" + t.text + "\"");
                    }
                    p.num.push_back(number(t));
                }
            };
            if (!first.quoted && first.text == "[") {
                for (;;) {
                    const Token& t = next(toks, i, decl);
                    if (!t.quoted && t.text == "]") break;
                    take(t);
                }
            } else {
                take(first);
            }
            ps.items.push_back(std::move(p));
        }
        ps.file = i > 0 ? files_[toks[i - 1].file] : std::string();
        return ps;
    }
};

class Parser : public Reader {
public:
    explicit Parser(ilm_scene_file* out) : out_(out) {}

    void run_file(const std::string& path) {
        std::ifstream f(path, std::ios::binary);
        if (!f) throw std::runtime_error(path + ": cannot open");
        std::stringstream ss;
        ss << f.rdbuf();
        run_text(ss.str(), path);
    }

    void run_text(const std::string& text, const std::string& name) {
        if (++depth_ > 16) throw std::runtime_error(name + ": Include nested more than 16 deep");
        files_.push_back(name);
        std::vector<Token> toks;
        tokenize(text, (int)files_.size() - 1, name, toks);
        size_t i = 0;
        while (i < toks.size()) directive(toks, i);
        --depth_;
    }

    void finish() {
        if (!stack_.empty()) warn_.push_back("AttributeBegin / TransformBegin without a matching end at end of input");
        if (in_object_) warn_.push_back("ObjectBegin without ObjectEnd at end of input");
        ilm_scene_file_info& in = out_->info;
        in.n_meshes = (uint32_t)out_->meshes.size();
        uint64_t nt = 0, nv = 0, ne = 0;
        for (const MeshOut& m : out_->meshes) {
            nt += m.idx.size() / 3;
            nv += m.xyz.size() / 3;
            const MaterialKey& k = out_->materials[m.material];
            if (k.emission[0] > 0 || k.emission[1] > 0 || k.emission[2] > 0) ne += m.idx.size() / 3;
        }
        if (nt + out_->quadrics.size() + out_->curves.size() >= (1ull << 28))
            throw std::runtime_error("more than 2^28 primitives");
        in.n_triangles = (uint32_t)nt;
        in.n_vertices = (uint32_t)nv;
        in.n_emissive = (uint32_t)ne;
        in.n_quadrics = (uint32_t)out_->quadrics.size();
        in.n_curves = (uint32_t)out_->curves.size();
        in.n_materials = (uint32_t)out_->materials.size();
        in.width = (uint32_t)width_;
        in.height = (uint32_t)height_;
        in.spp = spp_;
        in.max_depth = (uint32_t)max_depth_;
        // The camera: camera-to-world = inverse of the transform at Camera.
        const Mat4& c2w = camera_.inv;
        for (int k = 0; k < 3; ++k) in.eye[k] = (float)(c2w.m[k][3] / c2w.m[3][3]);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) in.camera_to_world[3 * r + c] = (float)c2w.m[r][c];
        // pbrt's fov spans the shorter image axis; the path tracer's spans y
        double half = fov_ * kPiD / 360.0;
        double vfov = width_ >= height_ ? fov_ : 2.0 * std::atan(std::tan(half) * height_ / width_) * 180.0 / kPiD;
        in.fov_deg = (float)vfov;
        in.filter = filter_;
        in.accelerator = kdtree_ ? 1 : 0;
        in.bvh = bvh_;
        in.kdtree = kd_;
        in.n_warnings = (uint32_t)warn_.size();
        for (const std::string& w : warn_) out_->warnings += w + "\n";
    }

private:

    void warn(const Token& t, const std::string& msg) { warn_.push_back(fname(t) + ":" + std::to_string(t.line) + ": " + msg); }

    void apply(const Xform& x) { st_.ctm = compose(st_.ctm, x); }

    uint32_t material_index(const GState& g) {
        MaterialKey k;
        for (int c = 0; c < 3; ++c) {
            k.albedo[c] = (float)g.kd[c];
            k.emission[c] = g.emits ? (float)g.le[c] : 0.0f;
        }
        auto it = mat_index_.find(k);
        if (it != mat_index_.end()) return it->second;
        uint32_t id = (uint32_t)out_->materials.size();
        out_->materials.push_back(k);
        mat_index_[k] = id;
        return id;
    }

    // Material "type" params (pbrt-v3 materials/*.cpp factories): matte's Kd
    // (0.5); other types keep their Kd when they have one.
    void set_material(const Token& t, const std::string& type, const Params& ps, GState& g) {
        double kd[3] = {0.5, 0.5, 0.5};
        if (type == "plastic" || type == "uber") kd[0] = kd[1] = kd[2] = 0.25;
        bool has = ps.rgb("Kd", kd, warn_);
        if (type != "matte")
            warn(t, "material \"" + type + "\" is shaded as matte" + (has ? " with its Kd" : " with Kd 0.5"));
        if (type == "matte") {
            ps.find("sigma", {"float"});
            ps.find("bumpmap", {"texture"});
        }
        for (int c = 0; c < 3; ++c) g.kd[c] = kd[c];
    }

    void emit_shape(const Token& t, const std::string& type, const Params& ps, const Xform& x, bool reverse,
                    uint32_t material) {
        ilm_sphere_desc q;
        std::memset(&q, 0, sizeof q);
        int kind = -1;
        if (type == "trianglemesh") {
            emit_mesh(t, ps, x, reverse, material);
            return;
        } else if (type == "loopsubdiv") {
            emit_loop(t, ps, x, reverse, material);
            return;
        } else if (type == "curve") {
            emit_curve(t, ps, x, reverse, material);
            return;
        } else if (type == "sphere") {
            kind = ILM_QUADRIC_SPHERE;
            q.radius = (float)ps.one_float("radius", 1.0);
            q.z_min = (float)ps.one_float("zmin", -q.radius);
            q.z_max = (float)ps.one_float("zmax", q.radius);
        } else if (type == "disk") {
            kind = ILM_QUADRIC_DISK;
            q.height = (float)ps.one_float("height", 0.0);
            q.radius = (float)ps.one_float("radius", 1.0);
            q.inner_radius = (float)ps.one_float("innerradius", 0.0);
        } else if (type == "cylinder") {
            kind = ILM_QUADRIC_CYLINDER;
            q.radius = (float)ps.one_float("radius", 1.0);
            q.z_min = (float)ps.one_float("zmin", -1.0);
            q.z_max = (float)ps.one_float("zmax", 1.0);
        } else if (type == "cone") {
            kind = ILM_QUADRIC_CONE;
            q.height = (float)ps.one_float("height", 1.0);
            q.radius = (float)ps.one_float("radius", 1.0);
        } else if (type == "paraboloid") {
            kind = ILM_QUADRIC_PARABOLOID;
            q.radius = (float)ps.one_float("radius", 1.0);
            q.z_min = (float)ps.one_float("zmin", 0.0);
            q.z_max = (float)ps.one_float("zmax", 1.0);
        } else if (type == "hyperboloid") {
            kind = ILM_QUADRIC_HYPERBOLOID;
            double p1[3] = {0, 0, 0}, p2[3] = {1, 1, 1};
            ps.point3("p1", p1);
            ps.point3("p2", p2);
            for (int k = 0; k < 3; ++k) { q.p1[k] = (float)p1[k]; q.p2[k] = (float)p2[k]; }
        } else {
            warn(t, "shape \"" + type + "\" is not supported; skipped");
            for (const Param& p : ps.items) p.used = true;
            return;
        }
        q.kind = kind;
        q.phi_max_deg = (float)ps.one_float("phimax", 360.0);
        q.reverse_orientation = reverse ? 1 : 0;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) {
                q.object_to_world[4 * r + c] = (float)x.m.m[r][c];
                q.world_to_object[4 * r + c] = (float)x.inv.m[r][c];
            }
        out_->quadrics.push_back(q);
        out_->quadric_material.push_back(material);
    }

    // Shape "curve" (pbrt-v3 CreateCurveShape): one cubic Bezier in object
    // space split into 2^splitdepth segments over equal u ranges.
    void emit_curve(const Token& t, const Params& ps, const Xform& x, bool reverse, uint32_t material) {
        const Param* P = ps.need_num("P", {"point"}, 3);
        if (!P || P->num.size() != 12) fail(t, "curve needs 4 control points in \"point P\"");
        double w = ps.one_float("width", 1.0);
        double w0 = ps.one_float("width0", w), w1 = ps.one_float("width1", w);
        if (!(w0 > 0 && w1 > 0)) fail(t, "curve widths must be positive");
        std::string type = ps.one_string("type", "flat");
        int ct = type == "flat" ? ILM_CURVE_FLAT : type == "cylinder" ? ILM_CURVE_CYLINDER
                 : type == "ribbon" ? ILM_CURVE_RIBBON : -1;
        if (ct < 0) {
            warn(t, "curve type \"" + type + "\" unknown; flat");
            ct = ILM_CURVE_FLAT;
        }
        const Param* N = ps.need_num("N", {"normal"}, 3);
        if (N && ct != ILM_CURVE_RIBBON) {
            warn(t, "curve normals are only used with ribbon curves");
            N = nullptr;
        }
        if (ct == ILM_CURVE_RIBBON && (!N || N->num.size() != 6)) fail(t, "ribbon curves need two normals in \"normal N\"");
        long sd = ps.one_int("splitdepth", 3);
        if (sd < 0 || sd > 10) fail(t, "splitdepth must be 0 .. 10");
        const int nseg = 1 << sd;
        for (int k = 0; k < nseg; ++k) {
            ilm_curve_desc c;
            std::memset(&c, 0, sizeof c);
            for (int r = 0; r < 4; ++r)
                for (int q = 0; q < 4; ++q) {
                    c.object_to_world[4 * r + q] = (float)x.m.m[r][q];
                    c.world_to_object[4 * r + q] = (float)x.inv.m[r][q];
                }
            for (int i = 0; i < 12; ++i) c.cp[i] = (float)P->num[i];
            c.width[0] = (float)w0;
            c.width[1] = (float)w1;
            if (N)
                for (int i = 0; i < 6; ++i) c.n[i] = (float)N->num[i];
            c.u_min = (float)k / (float)nseg;
            c.u_max = (float)(k + 1) / (float)nseg;
            c.type = ct;
            c.reverse_orientation = reverse ? 1 : 0;
            out_->curves.push_back(c);
            out_->curve_material.push_back(material);
        }
    }

    // Shape "loopsubdiv" (pbrt-v3 CreateLoopSubdiv): the control mesh
    // subdivided `levels` times (3), then placed like a trianglemesh with the
    // limit normals as N.
    void emit_loop(const Token& t, const Params& ps, const Xform& x, bool reverse, uint32_t material) {
        const Param* P = ps.need_num("P", {"point"}, 3);
        const Param* I = ps.need_num("indices", {"integer"}, 3);
        if (!P || !I) fail(t, "loopsubdiv needs \"point P\" and \"integer indices\"");
        long levels = ps.one_int("levels", ps.one_int("nlevels", 3));
        std::vector<float> p(P->num.begin(), P->num.end()), po, no;
        std::vector<uint32_t> idx, io;
        for (double v : I->num) {
            if (v < 0 || v >= (double)(P->num.size() / 3) || v != std::floor(v))
                fail_at(ps.file, I->line, "loopsubdiv index out of range");
            idx.push_back((uint32_t)v);
        }
        try {
            ilm::loop_subdivide(p, idx, (int)levels, po, io, no);
        } catch (const std::exception& e) {
            fail(t, e.what());
        }
        Params mesh;
        mesh.file = ps.file;
        Param pp, ip, np;
        pp.type = "point"; pp.name = "P"; pp.num.assign(po.begin(), po.end()); pp.line = t.line;
        ip.type = "integer"; ip.name = "indices"; ip.num.assign(io.begin(), io.end()); ip.line = t.line;
        np.type = "normal"; np.name = "N"; np.num.assign(no.begin(), no.end()); np.line = t.line;
        mesh.items = {pp, ip, np};
        emit_mesh(t, mesh, x, reverse, material);
    }

    // TriangleMesh::new (shapes/triangle.rs:36-73) with the Shape's transform
    // applied to P (points), S (vectors) and N (inverse transpose).
    void emit_mesh(const Token& t, const Params& ps, const Xform& x, bool reverse, uint32_t material) {
        const Param* P = ps.need_num("P", {"point"}, 3);
        if (!P) fail(t, "trianglemesh needs \"point P\"");
        const size_t nv = P->num.size() / 3;
        std::vector<uint32_t> idx;
        if (const Param* I = ps.need_num("indices", {"integer"}, 3)) {
            for (double v : I->num) {
                if (v < 0 || v >= (double)nv || v != std::floor(v)) fail_at(ps.file, I->line, "trianglemesh index out of range");
                idx.push_back((uint32_t)v);
            }
        } else if (nv == 3) {
            idx = {0, 1, 2};
        } else {
            fail(t, "trianglemesh needs \"integer indices\"");
        }
        MeshOut m;
        m.material = material;
        const Mat4& a = x.m;
        for (size_t i = 0; i < nv; ++i) {
            const double* p = &P->num[3 * i];
            double w = a.m[3][0] * p[0] + a.m[3][1] * p[1] + a.m[3][2] * p[2] + a.m[3][3];
            for (int r = 0; r < 3; ++r)
                m.xyz.push_back((float)((a.m[r][0] * p[0] + a.m[r][1] * p[1] + a.m[r][2] * p[2] + a.m[r][3]) / w));
        }
        if (const Param* N = ps.need_num("N", {"normal"}, 3)) {
            if (N->num.size() != 3 * nv) fail_at(ps.file, N->line, "\"normal N\" needs one normal per vertex");
            const Mat4& b = x.inv;
            for (size_t i = 0; i < nv; ++i) {
                const double* n = &N->num[3 * i];
                for (int c = 0; c < 3; ++c) m.n.push_back((float)(b.m[0][c] * n[0] + b.m[1][c] * n[1] + b.m[2][c] * n[2]));
            }
        }
        if (const Param* S = ps.need_num("S", {"vector"}, 3)) {
            if (S->num.size() != 3 * nv) fail_at(ps.file, S->line, "\"vector S\" needs one tangent per vertex");
            for (size_t i = 0; i < nv; ++i) {
                const double* s = &S->num[3 * i];
                for (int r = 0; r < 3; ++r) m.s.push_back((float)(a.m[r][0] * s[0] + a.m[r][1] * s[1] + a.m[r][2] * s[2]));
            }
        }
        const Param* UV = ps.need_num("uv", {"float", "point2"}, 2);
        if (!UV) UV = ps.need_num("st", {"float", "point2"}, 2);
        if (UV) {
            if (UV->num.size() != 2 * nv) fail_at(ps.file, UV->line, "\"uv\" needs one pair per vertex");
            for (double v : UV->num) m.uv.push_back((float)v);
        }
        for (const char* skip : {"alpha", "shadowalpha"})
            if (const Param* p = ps.find(skip, {"texture", "float"})) warn(t, std::string("\"") + p->name + "\" is not supported");
        // pbrt reports -n when ReverseOrientation and a handedness swap differ
        const bool flip = reverse != (det3(a) < 0.0);
        for (size_t k = 0; k + 2 < idx.size(); k += 3)
            if (flip) std::swap(idx[k + 1], idx[k + 2]);
        m.idx = std::move(idx);
        out_->meshes.push_back(std::move(m));
    }

    void directive(const std::vector<Token>& toks, size_t& i) { execute(read_directive(toks, i)); }

    void execute(const Directive& D) {
        const Token& d = D.tok;
        const std::string& n = d.text;
        const std::vector<double>& v = D.num;
        const Params& ps = D.params;
        auto done = [&](const Params& ps, const std::string& what) { ps.report_unused(what, warn_); };
        if (n == "Identity") {
            st_.ctm = Xform();
        } else if (n == "Translate") {
            apply(translate(v[0], v[1], v[2]));
        } else if (n == "Scale") {
            if (v[0] == 0 || v[1] == 0 || v[2] == 0) fail(d, "Scale by zero");
            apply(scale(v[0], v[1], v[2]));
        } else if (n == "Rotate") {
            if (v[1] == 0 && v[2] == 0 && v[3] == 0) fail(d, "Rotate about a zero axis");
            apply(rotate(v[0], v[1], v[2], v[3]));
        } else if (n == "LookAt") {
            Xform la;
            if (!look_at(&v[0], &v[3], &v[6], &la)) warn(d, "LookAt with up parallel to the view direction; ignored");
            else apply(la);
        } else if (n == "Transform" || n == "ConcatTransform") {
            // 16 numbers, the matrix's columns (pbrt-v3 transposes them)
            Mat4 m;
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) m.m[c][r] = v[4 * r + c];
            Mat4 inv;
            if (!invert4(m, &inv)) fail(d, n + " matrix is singular");
            Xform x{m, inv};
            if (n == "Transform") st_.ctm = x;
            else apply(x);
        } else if (n == "CoordinateSystem") {
            named_[D.str[0]] = st_.ctm;
        } else if (n == "CoordSysTransform") {
            const std::string& name = D.str[0];
            auto it = named_.find(name);
            if (it == named_.end()) warn(d, "coordinate system \"" + name + "\" not declared; ignored");
            else st_.ctm = it->second;
        } else if (n == "ActiveTransform") {
            if (D.str[0] != "All") warn(d, "motion transforms are not supported; both times get every transform");
        } else if (n == "TransformTimes") {
            warn(d, "TransformTimes ignored (no motion blur)");
        } else if (n == "ReverseOrientation") {
            st_.reverse = !st_.reverse;
        } else if (n == "WorldBegin") {
            st_.ctm = Xform();
            named_["world"] = st_.ctm;
            in_world_ = true;
        } else if (n == "WorldEnd") {
            in_world_ = false;
        } else if (n == "AttributeBegin" || n == "TransformBegin") {
            stack_.push_back({st_, n == "TransformBegin"});
        } else if (n == "AttributeEnd" || n == "TransformEnd") {
            if (stack_.empty()) fail(d, "unmatched " + n);
            Frame f = stack_.back();
            stack_.pop_back();
            if (f.transform_only != (n == "TransformEnd")) fail(d, n + " closes a block opened by the other kind");
            if (f.transform_only) st_.ctm = f.state.ctm;
            else st_ = f.state;
        } else if (n == "ObjectBegin") {
            const std::string& name = D.str[0];
            if (in_object_) fail(d, "ObjectBegin inside an object");
            stack_.push_back({st_, false});
            in_object_ = true;
            object_ = name;
            objects_[name].clear();
        } else if (n == "ObjectEnd") {
            if (!in_object_) fail(d, "ObjectEnd without ObjectBegin");
            in_object_ = false;
            if (stack_.empty()) fail(d, "unmatched ObjectEnd");
            st_ = stack_.back().state;
            stack_.pop_back();
        } else if (n == "ObjectInstance") {
            const std::string& name = D.str[0];
            auto it = objects_.find(name);
            if (it == objects_.end()) fail(d, "object \"" + name + "\" not defined");
            for (const ShapeRecord& r : it->second)
                emit_shape(d, r.type, r.params, compose(st_.ctm, r.ctm), r.reverse, r.material);
        } else if (n == "Shape") {
            const std::string& type = D.str[0];
            if (in_object_) {
                if (st_.emits) warn(d, "area lights inside object instances are not supported; shape not emissive");
                GState g = st_;
                g.emits = false;
                objects_[object_].push_back({type, ps, st_.ctm, st_.reverse, material_index(g), d.line});
                for (const Param& p : ps.items) p.used = true;
            } else {
                emit_shape(d, type, ps, st_.ctm, st_.reverse, material_index(st_));
                done(ps, "shape \"" + type + "\"");
            }
        } else if (n == "Material") {
            const std::string& type = D.str[0];
            set_material(d, type, ps, st_);
            done(ps, "material \"" + type + "\"");
        } else if (n == "MakeNamedMaterial") {
            const std::string& name = D.str[0];
            std::string type = ps.one_string("type", "");
            if (type.empty()) fail(d, "MakeNamedMaterial needs \"string type\"");
            GState g;
            set_material(d, type, ps, g);
            std::copy(g.kd, g.kd + 3, named_mats_[name].kd);
            done(ps, "material \"" + name + "\"");
        } else if (n == "NamedMaterial") {
            const std::string& name = D.str[0];
            auto it = named_mats_.find(name);
            if (it == named_mats_.end()) fail(d, "named material \"" + name + "\" not defined");
            std::copy(it->second.kd, it->second.kd + 3, st_.kd);
        } else if (n == "AreaLightSource") {
            const std::string& type = D.str[0];
            if (type != "diffuse") {
                warn(d, "area light \"" + type + "\" is not supported; shapes stay non-emissive");
                for (const Param& p : ps.items) p.used = true;
            } else {
                // CreateDiffuseAreaLight (pbrt-v3): L x scale, one-sided
                double L[3] = {1, 1, 1}, sc[3] = {1, 1, 1};
                ps.rgb("L", L, warn_);
                ps.rgb("scale", sc, warn_);
                if (ps.one_bool("twosided", false)) warn(d, "two-sided area lights emit on one side here");
                ps.one_int("samples", 1);
                ps.one_int("nsamples", 1);
                st_.emits = true;
                for (int c = 0; c < 3; ++c) st_.le[c] = L[c] * sc[c];
                done(ps, "area light");
            }
        } else if (n == "LightSource") {
            const std::string& type = D.str[0];
            for (const Param& p : ps.items) p.used = true;
            warn(d, "light \"" + type + "\" is not supported (area lights only); skipped");
        } else if (n == "Camera") {
            const std::string& type = D.str[0];
            if (type != "perspective") warn(d, "camera \"" + type + "\" is rendered as a perspective camera");
            camera_ = st_.ctm;
            named_["camera"] = Xform{st_.ctm.inv, st_.ctm.m};
            double half = ps.one_float("halffov", -1.0);
            fov_ = ps.one_float("fov", half > 0 ? 2.0 * half : 90.0);
            if (!(fov_ > 0.0 && fov_ < 180.0)) fail(d, "camera fov must lie in (0, 180)");
            if (ps.one_float("lensradius", 0.0) > 0.0) warn(d, "lens radius ignored (pinhole camera)");
            ps.one_float("focaldistance", 1e6);
            ps.one_float("frameaspectratio", 0.0);
            if (ps.find("screenwindow", {"float"})) warn(d, "screenwindow ignored");
            ps.one_float("shutteropen", 0.0);
            ps.one_float("shutterclose", 1.0);
            done(ps, "camera");
        } else if (n == "Film") {
            width_ = ps.one_int("xresolution", 640);
            height_ = ps.one_int("yresolution", 480);
            if (width_ <= 0 || height_ <= 0 || width_ > 65536 || height_ > 65536) fail(d, "film resolution out of range");
            ps.one_string("filename", "");
            if (ps.find("cropwindow", {"float"})) warn(d, "cropwindow ignored");
            ps.one_float("diagonal", 35.0);
            ps.one_float("scale", 1.0);
            ps.one_float("maxsampleluminance", INFINITY);
            done(ps, "film");
        } else if (n == "Sampler") {
            const std::string& type = D.str[0];
            long want;
            if (type == "stratified") {
                want = ps.one_int("xsamples", 4) * ps.one_int("ysamples", 4);
                ps.one_bool("jitter", true);
            } else {
                want = ps.one_int("pixelsamples", type == "random" ? 4 : 16);
            }
            if (want <= 0) fail(d, "sampler needs a positive sample count");
            long ns = (long)std::ceil(std::sqrt((double)want));
            if (ns * ns != want) warn(d, "samples per pixel rounded up to " + std::to_string(ns * ns) + " (a square)");
            spp_ = (uint32_t)(ns * ns);
            ps.one_int("dimensions", 4);
            done(ps, "sampler");
        } else if (n == "Integrator") {
            const std::string& type = D.str[0];
            if (type != "path") warn(d, "integrator \"" + type + "\" is rendered by the path integrator");
            max_depth_ = ps.one_int("maxdepth", 5);
            if (max_depth_ < 0) fail(d, "maxdepth must be non-negative");
            ps.one_float("rrthreshold", 1.0);
            ps.one_string("lightsamplestrategy", "spatial");
            if (ps.find("pixelbounds", {"integer"})) warn(d, "pixelbounds ignored");
            done(ps, "integrator");
        } else if (n == "PixelFilter") {
            const std::string& type = D.str[0];
            ilm_filter_desc f{};
            double w = type == "box" ? 0.5 : (type == "sinc" ? 4.0 : 2.0);
            f.radius[0] = (float)ps.one_float("xwidth", w);
            f.radius[1] = (float)ps.one_float("ywidth", w);
            if (type == "box") f.kind = ILM_FILTER_BOX;
            else if (type == "triangle") f.kind = ILM_FILTER_TRIANGLE;
            else if (type == "gaussian") { f.kind = ILM_FILTER_GAUSSIAN; f.a = (float)ps.one_float("alpha", 2.0); }
            else if (type == "mitchell") {
                f.kind = ILM_FILTER_MITCHELL;
                f.a = (float)ps.one_float("B", 1.0 / 3.0);
                f.b = (float)ps.one_float("C", 1.0 / 3.0);
            } else if (type == "sinc") { f.kind = ILM_FILTER_LANCZOS; f.a = (float)ps.one_float("tau", 3.0); }
            else fail(d, "unknown pixel filter \"" + type + "\"");
            if (!(f.radius[0] > 0 && f.radius[1] > 0)) fail(d, "filter widths must be positive");
            filter_ = f;
            done(ps, "filter");
        } else if (n == "Accelerator") {
            const std::string& type = D.str[0];
            if (type == "bvh") {
                kdtree_ = false;
                bvh_.max_prims_in_node = (int32_t)std::min(255L, ps.one_int("maxnodeprims", 4));
                std::string sm = ps.one_string("splitmethod", "sah");
                if (sm != "sah") warn(d, "split method \"" + sm + "\" is built as sah");
            } else if (type == "kdtree") {
                kdtree_ = true;
                kd_.isect_cost = (int32_t)ps.one_int("intersectcost", 80);
                kd_.traversal_cost = (int32_t)ps.one_int("traversalcost", 1);
                kd_.empty_bonus = (float)ps.one_float("emptybonus", 0.5);
                kd_.max_prims = (uint32_t)std::max(0L, ps.one_int("maxprims", 1));
                kd_.max_depth = (int32_t)ps.one_int("maxdepth", -1);
            } else {
                warn(d, "accelerator \"" + type + "\" is built as a bvh");
            }
            done(ps, "accelerator");
        } else if (n == "Texture") {
            const std::string& cls = D.str[2];
            for (const Param& p : ps.items) p.used = true;
            warn(d, "texture \"" + cls + "\" is not supported; materials use their constant defaults");
        } else if (n == "MakeNamedMedium" || n == "MediumInterface") {
            for (const Param& p : ps.items) p.used = true;
            warn(d, "participating media are not supported; " + n + " skipped");
        } else if (n == "Include") {
            const std::string& path = D.str[0];
            std::string dir = fname(d);
            size_t cut = dir.find_last_of('/');
            std::string base = cut == std::string::npos ? base_dir_ : dir.substr(0, cut);
            std::string full = !path.empty() && path[0] == '/' ? path : (base.empty() ? path : base + "/" + path);
            run_file(full);
        } else {
            fail(d, "unknown directive \"" + n + "\"");
        }
    }

    struct Frame {
        GState state;
        bool transform_only;
    };
    struct NamedMat {
        double kd[3];
    };

    ilm_scene_file* out_;
    std::vector<std::string> warn_;
    int depth_ = 0;
    GState st_;
    std::vector<Frame> stack_;
    std::map<std::string, Xform> named_;
    std::map<std::string, NamedMat> named_mats_;
    std::map<std::string, std::vector<ShapeRecord>> objects_;
    std::map<MaterialKey, uint32_t> mat_index_;
    bool in_object_ = false, in_world_ = false;
    std::string object_;
    Xform camera_;
    double fov_ = 90.0;
    long width_ = 640, height_ = 480;
    uint32_t spp_ = 16;
    long max_depth_ = 5;
    ilm_filter_desc filter_{ILM_FILTER_BOX, {0.5f, 0.5f}, 0.0f, 0.0f};
    bool kdtree_ = false;
    ilm_build_opts bvh_{8, 4};
    ilm_kdtree_opts kd_{80, 1, 0.5f, 1, -1};

public:
    std::string base_dir_;
};

int32_t finish_load(Parser& p, std::unique_ptr<ilm_scene_file>& sf, ilm_scene_file** out) {
    p.finish();
    *out = sf.release();
    return ILM_OK;
}

void put_error(char* error, size_t error_len, const std::string& msg) {
    if (!error || error_len == 0) return;
    std::snprintf(error, error_len, "%s", msg.c_str());
}

// ------------------------------------------------------------ syntax dump
// The directive tree of a scene description, read with the loader's tokenizer
// and Reader::read_directive but not run: the tree parse_to_ast returns
// (core/parser/mod.rs:19-34).  AttributeBegin, TransformBegin, ObjectBegin and
// WorldBegin open a block that holds the directives up to its matching end
// (ast.rs's Attribute, Transform, Object and World directives); Include is
// replaced by the directives of the file it names (many_with_include,
// core/parser/parsers/directives.rs).
class SyntaxDump : public Reader {
public:
    std::string base_dir_;

    std::string run(const std::string& text) {
        std::vector<Node> top;
        std::vector<Block> open;
        read_text(text, "<text>", top, open);
        if (!open.empty()) {
            const Node& b = open.back().node;
            fail(b.d.tok, b.d.tok.text + " without a matching end");
        }
        std::string out = "{\"directives\":";
        list(top, out);
        out += ",\"comments\":[";
        for (size_t k = 0; k < comments_.size(); ++k) {
            if (k) out += ',';
            str(comments_[k], out);
        }
        out += "]}";
        return out;
    }

private:
    struct Node {
        Directive d;
        bool block = false;
        std::vector<Node> children;
    };
    struct Block {
        Node node;
        std::string end;
    };

    std::vector<std::string> comments_;
    int depth_ = 0;

    void read_text(const std::string& text, const std::string& name, std::vector<Node>& top, std::vector<Block>& open) {
        if (++depth_ > 16) throw std::runtime_error(name + ": Include nested more than 16 deep");
        files_.push_back(name);
        std::vector<Token> toks;
        tokenize(text, (int)files_.size() - 1, name, toks, &comments_);
        size_t i = 0;
        while (i < toks.size()) {
            Node n;
            n.d = read_directive(toks, i);
            const std::string& w = n.d.tok.text;
            static const std::map<std::string, std::string> ends = {{"AttributeBegin", "AttributeEnd"},
                                                                    {"TransformBegin", "TransformEnd"},
                                                                    {"ObjectBegin", "ObjectEnd"},
                                                                    {"WorldBegin", "WorldEnd"}};
            auto e = ends.find(w);
            if (e != ends.end()) {
                n.block = true;
                open.push_back({std::move(n), e->second});
            } else if (w == "AttributeEnd" || w == "TransformEnd" || w == "ObjectEnd" || w == "WorldEnd") {
                if (open.empty() || open.back().end != w) fail(n.d.tok, "unmatched " + w);
                Node b = std::move(open.back().node);
                open.pop_back();
                (open.empty() ? top : open.back().node.children).push_back(std::move(b));
            } else if (w == "Include") {
                std::string dir = fname(n.d.tok);
                size_t cut = dir.find_last_of('/');
                std::string base = cut == std::string::npos ? base_dir_ : dir.substr(0, cut);
                const std::string& path = n.d.str[0];
                std::string full = !path.empty() && path[0] == '/' ? path : (base.empty() ? path : base + "/" + path);
                std::ifstream f(full, std::ios::binary);
                if (!f) throw std::runtime_error(full + ": cannot open");
                std::stringstream ss;
                ss << f.rdbuf();
                read_text(ss.str(), full, top, open);
            } else {
                (open.empty() ? top : open.back().node.children).push_back(std::move(n));
            }
        }
        --depth_;
    }

    static void str(const std::string& v, std::string& out) {
        out += '"';
        for (unsigned char c : v) {
            if (c == '"' || c == '\\') {
                out += '\\';
                out += (char)c;
            } else if (c < 0x20) {
                char buf[8];
                std::snprintf(buf, sizeof buf, "\\u%04x", c);
                out += buf;
            } else {
                out += (char)c;
            }
        }
        out += '"';
    }
    static void nums(const std::vector<double>& v, std::string& out) {
        out += '[';
        for (size_t k = 0; k < v.size(); ++k) {
            char buf[32];
            std::snprintf(buf, sizeof buf, "%s%.17g", k ? "," : "", v[k]);
            out += buf;
        }
        out += ']';
    }
    static void strs(const std::vector<std::string>& v, std::string& out) {
        out += '[';
        for (size_t k = 0; k < v.size(); ++k) {
            if (k) out += ',';
            str(v[k], out);
        }
        out += ']';
    }
    void node(const Node& n, std::string& out) const {
        out += "{\"directive\":";
        str(n.d.tok.text, out);
        out += ",\"file\":";
        str(fname(n.d.tok), out);
        out += ",\"line\":" + std::to_string(n.d.tok.line) + ",\"num\":";
        nums(n.d.num, out);
        out += ",\"str\":";
        strs(n.d.str, out);
        out += ",\"params\":[";
        for (size_t k = 0; k < n.d.params.items.size(); ++k) {
            const Param& p = n.d.params.items[k];
            if (k) out += ',';
            out += "{\"type\":";
            str(p.type, out);
            out += ",\"name\":";
            str(p.name, out);
            out += ",\"num\":";
            nums(p.num, out);
            out += ",\"str\":";
            strs(p.str, out);
            out += '}';
        }
        out += ']';
        if (n.block) {
            out += ",\"children\":";
            list(n.children, out);
        }
        out += '}';
    }
    void list(const std::vector<Node>& v, std::string& out) const {
        out += '[';
        for (size_t k = 0; k < v.size(); ++k) {
            if (k) out += ',';
            node(v[k], out);
        }
        out += ']';
    }
};

}  // namespace

extern "C" {

int32_t ilm_scene_file_load(const char* path, char* error, size_t error_len, ilm_scene_file** out) {
    if (!out || !path) return ILM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto sf = std::make_unique<ilm_scene_file>();
    Parser p(sf.get());
    try {
        std::string s(path);
        size_t cut = s.find_last_of('/');
        p.base_dir_ = cut == std::string::npos ? std::string() : s.substr(0, cut);
        p.run_file(s);
        return finish_load(p, sf, out);
    } catch (const std::exception& e) {
        put_error(error, error_len, e.what());
        return ILM_ERR_INVALID_ARGUMENT;
    }
}

int32_t ilm_scene_file_parse(const char* text, const char* base_dir, char* error, size_t error_len,
                             ilm_scene_file** out) {
    if (!out || !text) return ILM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto sf = std::make_unique<ilm_scene_file>();
    Parser p(sf.get());
    try {
        p.base_dir_ = base_dir ? base_dir : "";
        p.run_text(text, "<text>");
        return finish_load(p, sf, out);
    } catch (const std::exception& e) {
        put_error(error, error_len, e.what());
        return ILM_ERR_INVALID_ARGUMENT;
    }
}

int32_t ilm_scene_syntax(const char* text, const char* base_dir, char* json, size_t json_cap, size_t* json_len,
                         char* error, size_t error_len) {
    if (!text || !json_len || (json_cap && !json)) return ILM_ERR_INVALID_ARGUMENT;
    try {
        SyntaxDump d;
        d.base_dir_ = base_dir ? base_dir : "";
        std::string out = d.run(text);
        *json_len = out.size();
        if (json_cap) {
            size_t k = std::min(out.size(), json_cap - 1);
            std::memcpy(json, out.data(), k);
            json[k] = '\0';
        }
        return ILM_OK;
    } catch (const std::exception& e) {
        put_error(error, error_len, e.what());
        return ILM_ERR_INVALID_ARGUMENT;
    }
}

int32_t ilm_scene_file_info_get(const ilm_scene_file* sf, ilm_scene_file_info* out) {
    if (!sf || !out) return ILM_ERR_INVALID_ARGUMENT;
    *out = sf->info;
    return ILM_OK;
}

const char* ilm_scene_file_warnings(const ilm_scene_file* sf) { return sf ? sf->warnings.c_str() : ""; }

int32_t ilm_scene_file_mesh(const ilm_scene_file* sf, uint32_t k, uint32_t* nv, uint32_t* nt, float* xyz,
                            uint32_t* idx, float* n, float* s, float* uv, int32_t* has_n, int32_t* has_s,
                            int32_t* has_uv, uint32_t* material) {
    if (!sf || k >= sf->meshes.size()) return ILM_ERR_INVALID_ARGUMENT;
    const MeshOut& m = sf->meshes[k];
    if (nv) *nv = (uint32_t)(m.xyz.size() / 3);
    if (nt) *nt = (uint32_t)(m.idx.size() / 3);
    auto put = [](const auto& v, auto* dst) { if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0])); };
    put(m.xyz, xyz);
    put(m.idx, idx);
    put(m.n, n);
    put(m.s, s);
    put(m.uv, uv);
    if (has_n) *has_n = !m.n.empty();
    if (has_s) *has_s = !m.s.empty();
    if (has_uv) *has_uv = !m.uv.empty();
    if (material) *material = m.material;
    return ILM_OK;
}

int32_t ilm_scene_file_quadrics(const ilm_scene_file* sf, ilm_sphere_desc* out, uint32_t* material) {
    if (!sf) return ILM_ERR_INVALID_ARGUMENT;
    if (out && !sf->quadrics.empty()) std::memcpy(out, sf->quadrics.data(), sf->quadrics.size() * sizeof(ilm_sphere_desc));
    if (material && !sf->quadric_material.empty())
        std::memcpy(material, sf->quadric_material.data(), sf->quadric_material.size() * 4);
    return ILM_OK;
}

int32_t ilm_scene_file_curves(const ilm_scene_file* sf, ilm_curve_desc* out, uint32_t* material) {
    if (!sf) return ILM_ERR_INVALID_ARGUMENT;
    if (out && !sf->curves.empty()) std::memcpy(out, sf->curves.data(), sf->curves.size() * sizeof(ilm_curve_desc));
    if (material && !sf->curve_material.empty())
        std::memcpy(material, sf->curve_material.data(), sf->curve_material.size() * 4);
    return ILM_OK;
}

int32_t ilm_scene_file_materials(const ilm_scene_file* sf, float* albedo, float* emission) {
    if (!sf) return ILM_ERR_INVALID_ARGUMENT;
    for (size_t i = 0; i < sf->materials.size(); ++i)
        for (int c = 0; c < 3; ++c) {
            if (albedo) albedo[3 * i + c] = sf->materials[i].albedo[c];
            if (emission) emission[3 * i + c] = sf->materials[i].emission[c];
        }
    return ILM_OK;
}

int32_t ilm_scene_file_build(ilm_context* ctx, const ilm_scene_file* sf, ilm_accel_id* accel_out,
                             ilm_pt_scene_id* pt_out) {
    if (!ctx || !sf || !accel_out) return ILM_ERR_INVALID_ARGUMENT;
    if (pt_out) *pt_out = 0;
    std::vector<ilm_mesh_id> ids;
    std::vector<uint32_t> prim_material;
    int32_t rc;
    for (const MeshOut& m : sf->meshes) {
        ilm_mesh_id id;
        if ((rc = ilm_mesh_upload(ctx, m.xyz.data(), (uint32_t)(m.xyz.size() / 3), m.idx.data(),
                                  (uint32_t)(m.idx.size() / 3), &id)) != ILM_OK)
            return rc;
        if (!m.n.empty() || !m.s.empty() || !m.uv.empty()) {
            ilm_mesh_attrs a{m.n.empty() ? nullptr : m.n.data(), m.s.empty() ? nullptr : m.s.data(),
                             m.uv.empty() ? nullptr : m.uv.data(), 0};
            if ((rc = ilm_mesh_set_attrs(ctx, id, &a)) != ILM_OK) return rc;
        }
        ids.push_back(id);
        prim_material.insert(prim_material.end(), m.idx.size() / 3, m.material);
    }
    if (!sf->quadrics.empty()) {
        ilm_mesh_id id;
        if ((rc = ilm_spheres_upload(ctx, sf->quadrics.data(), (uint32_t)sf->quadrics.size(), &id)) != ILM_OK) return rc;
        ids.push_back(id);
    }
    if (!sf->curves.empty()) {
        ilm_mesh_id id;
        if ((rc = ilm_curves_upload(ctx, sf->curves.data(), (uint32_t)sf->curves.size(), &id)) != ILM_OK) return rc;
        ids.push_back(id);
    }
    const ilm_scene_file_info& in = sf->info;
    rc = in.accelerator == 1 ? ilm_kdtree_build(ctx, ids.data(), (uint32_t)ids.size(), &in.kdtree, accel_out)
                             : ilm_accel_build(ctx, ids.data(), (uint32_t)ids.size(), &in.bvh, accel_out);
    if (rc != ILM_OK) return rc;
    if (!pt_out || !sf->quadrics.empty() || !sf->curves.empty() || sf->meshes.empty()) return ILM_OK;
    std::vector<float> albedo(3 * sf->materials.size()), emission(3 * sf->materials.size());
    ilm_scene_file_materials(sf, albedo.data(), emission.data());
    ilm_pt_scene_desc d;
    std::memset(&d, 0, sizeof d);
    d.prim_material = prim_material.data();
    d.albedo = albedo.data();
    d.emission = emission.data();
    d.n_materials = (uint32_t)sf->materials.size();
    std::memcpy(d.eye, in.eye, sizeof d.eye);
    d.fov_deg = in.fov_deg;
    d.width = in.width;
    d.height = in.height;
    std::memcpy(d.camera_to_world, in.camera_to_world, sizeof d.camera_to_world);
    return ilm_pt_scene_create(ctx, *accel_out, &d, pt_out);
}

int32_t ilm_loop_subdivide(const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt, uint32_t levels,
                           uint32_t* out_nv, uint32_t* out_nt, float* out_xyz, uint32_t* out_idx, float* out_n) {
    if ((nv && !xyz) || (nt && !idx) || !out_nv || !out_nt) return ILM_ERR_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < 3ull * nv; ++i)
        if (!std::isfinite(xyz[i])) return ILM_ERR_INVALID_ARGUMENT;
    std::vector<float> p(xyz, xyz + 3ull * nv), po, no;
    std::vector<uint32_t> ix(idx, idx + 3ull * nt), io;
    try {
        ilm::loop_subdivide(p, ix, (int)levels, po, io, no);
    } catch (const std::exception&) {
        return ILM_ERR_INVALID_ARGUMENT;
    }
    const uint32_t onv = (uint32_t)(po.size() / 3), ont = (uint32_t)(io.size() / 3);
    if (out_xyz) {
        if (*out_nv < onv || *out_nt < ont) return ILM_ERR_INVALID_ARGUMENT;
        std::memcpy(out_xyz, po.data(), po.size() * 4);
        if (out_idx) std::memcpy(out_idx, io.data(), io.size() * 4);
        if (out_n) std::memcpy(out_n, no.data(), no.size() * 4);
    }
    *out_nv = onv;
    *out_nt = ont;
    return ILM_OK;
}

int32_t ilm_scene_file_destroy(ilm_scene_file* sf) {
    if (!sf) return ILM_ERR_INVALID_ARGUMENT;
    delete sf;
    return ILM_OK;
}

}  // extern "C"
