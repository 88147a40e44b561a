// Oracle (test infrastructure only): XML scene loading (parser.cpp:41-235), OBJ
// loading (mesh.cpp:148-229) and the transform factories (transform.h:388-431),
// restated without pugixml, tinyobjloader or glm.
#include "oscene.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <thread>
#include <unordered_map>

namespace orc {

// ---------------------------------------------------------------- matrices
Mat4 Inverse(const Mat4& mm) {
    // Cofactor expansion on the row-major copy a[r][c].
    float a[4][4];
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) a[r][c] = mm.c[c][r];
    float inv[4][4];
    for (int r = 0; r < 4; ++r) {
        for (int c = 0; c < 4; ++c) {
            float sub[3][3];
            int si = 0;
            for (int i = 0; i < 4; ++i) {
                if (i == c) continue;
                int sj = 0;
                for (int j = 0; j < 4; ++j) {
                    if (j == r) continue;
                    sub[si][sj++] = a[i][j];
                }
                ++si;
            }
            float det3 = sub[0][0] * (sub[1][1] * sub[2][2] - sub[1][2] * sub[2][1]) -
                         sub[0][1] * (sub[1][0] * sub[2][2] - sub[1][2] * sub[2][0]) +
                         sub[0][2] * (sub[1][0] * sub[2][1] - sub[1][1] * sub[2][0]);
            inv[r][c] = ((r + c) & 1) ? -det3 : det3;
        }
    }
    float det = a[0][0] * inv[0][0] + a[0][1] * inv[1][0] + a[0][2] * inv[2][0] + a[0][3] * inv[3][0];
    float invDet = 1.0f / det;
    Mat4 out;
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) out.c[c][r] = inv[r][c] * invDet;
    return out;
}

Transform Transform::Translate(const Vec3& d) {
    Mat4 m, mi;
    m.c[3][0] = d.x; m.c[3][1] = d.y; m.c[3][2] = d.z;
    mi.c[3][0] = -d.x; mi.c[3][1] = -d.y; mi.c[3][2] = -d.z;
    return Transform(m, mi);
}
Transform Transform::Scale(float x, float y, float z) {
    Mat4 m, mi;
    m.c[0][0] = x; m.c[1][1] = y; m.c[2][2] = z;
    mi.c[0][0] = 1.f / x; mi.c[1][1] = 1.f / y; mi.c[2][2] = 1.f / z;
    return Transform(m, mi);
}
// Rodrigues rotation about a normalised axis (the matrix glm::rotate builds); the
// inverse is the transpose (transform.h:421-426).
Transform Transform::Rotate(float degrees, const Vec3& axisIn) {
    float rad = degrees * 0.01745329251994329576923690768489f;
    float c = std::cos(rad), s = std::sin(rad);
    Vec3 ax = Normalize(axisIn);
    Vec3 tmp = ax * (1.0f - c);
    Mat4 m;
    m.c[0][0] = c + tmp.x * ax.x;
    m.c[0][1] = tmp.x * ax.y + s * ax.z;
    m.c[0][2] = tmp.x * ax.z - s * ax.y;
    m.c[1][0] = tmp.y * ax.x - s * ax.z;
    m.c[1][1] = c + tmp.y * ax.y;
    m.c[1][2] = tmp.y * ax.z + s * ax.x;
    m.c[2][0] = tmp.z * ax.x + s * ax.y;
    m.c[2][1] = tmp.z * ax.y - s * ax.x;
    m.c[2][2] = c + tmp.z * ax.z;
    return Transform(m, m.transpose());
}
// Right-handed look-at view matrix; camera-to-world is its inverse (transform.h:428-431).
Transform Transform::LookAt(const Vec3& pos, const Vec3& target, const Vec3& up) {
    Vec3 f = Normalize(target - pos);
    Vec3 s = Normalize(Cross(f, up));
    Vec3 u = Cross(s, f);
    Mat4 v;
    v.c[0][0] = s.x; v.c[1][0] = s.y; v.c[2][0] = s.z;
    v.c[0][1] = u.x; v.c[1][1] = u.y; v.c[2][1] = u.z;
    v.c[0][2] = -f.x; v.c[1][2] = -f.y; v.c[2][2] = -f.z;
    v.c[3][0] = -Dot(s, pos); v.c[3][1] = -Dot(u, pos); v.c[3][2] = Dot(f, pos);
    return Transform(Inverse(v), v);
}

// ---------------------------------------------------------------- minimal XML
namespace {
struct XNode {
    std::string tag;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XNode> kids;
    const char* attr(const char* k) const {
        for (auto& a : attrs) if (a.first == k) return a.second.c_str();
        return nullptr;
    }
};

struct XParser {
    const std::string& s;
    size_t i = 0;
    explicit XParser(const std::string& src) : s(src) {}
    [[noreturn]] void fail(const std::string& m) { throw std::runtime_error("XML parsing failed: " + m); }
    void skipWs() { while (i < s.size() && isspace((unsigned char)s[i])) ++i; }
    void skipMisc() {
        for (;;) {
            skipWs();
            if (s.compare(i, 4, "<!--") == 0) { size_t e = s.find("-->", i); if (e == std::string::npos) fail("unterminated comment"); i = e + 3; }
            else if (s.compare(i, 2, "<?") == 0) { size_t e = s.find("?>", i); if (e == std::string::npos) fail("unterminated declaration"); i = e + 2; }
            else if (s.compare(i, 2, "<!") == 0) { size_t e = s.find('>', i); if (e == std::string::npos) fail("bad markup"); i = e + 1; }
            else break;
        }
    }
    static std::string unescape(const std::string& v) {
        std::string o;
        for (size_t k = 0; k < v.size(); ++k) {
            if (v[k] == '&') {
                size_t e = v.find(';', k);
                std::string ent = v.substr(k + 1, e - k - 1);
                if (ent == "amp") o += '&'; else if (ent == "lt") o += '<'; else if (ent == "gt") o += '>';
                else if (ent == "quot") o += '"'; else if (ent == "apos") o += '\''; else o += "&" + ent + ";";
                k = e;
            } else o += v[k];
        }
        return o;
    }
    std::string name() {
        size_t st = i;
        while (i < s.size() && (isalnum((unsigned char)s[i]) || s[i] == '_' || s[i] == '-' || s[i] == ':' || s[i] == '.')) ++i;
        if (st == i) fail("expected a name at offset " + std::to_string(st));
        return s.substr(st, i - st);
    }
    XNode element() {
        if (s[i] != '<') fail("expected '<' at offset " + std::to_string(i));
        ++i;
        XNode n;
        n.tag = name();
        for (;;) {
            skipWs();
            if (i >= s.size()) fail("unterminated tag <" + n.tag + ">");
            if (s[i] == '/') { if (s[i + 1] != '>') fail("bad '/'"); i += 2; return n; }
            if (s[i] == '>') { ++i; break; }
            std::string k = name();
            skipWs();
            if (s[i] != '=') fail("expected '=' after attribute " + k);
            ++i; skipWs();
            char q = s[i];
            if (q != '"' && q != '\'') fail("expected quote");
            size_t e = s.find(q, i + 1);
            if (e == std::string::npos) fail("unterminated attribute");
            n.attrs.push_back({k, unescape(s.substr(i + 1, e - i - 1))});
            i = e + 1;
        }
        for (;;) {
            size_t lt = s.find('<', i);
            if (lt == std::string::npos) fail("missing </" + n.tag + ">");
            i = lt;
            if (s.compare(i, 4, "<!--") == 0 || s.compare(i, 2, "<?") == 0) { skipMisc(); continue; }
            if (s.compare(i, 2, "</") == 0) {
                i += 2;
                std::string nm = name();
                if (nm != n.tag) fail("mismatched </" + nm + "> for <" + n.tag + ">");
                skipWs();
                if (s[i] != '>') fail("bad closing tag");
                ++i;
                return n;
            }
            n.kids.push_back(element());
        }
    }
};

float asFloat(const char* v, float d) { if (!v || !*v) return d; return (float)std::strtod(v, nullptr); }
int asInt(const char* v, int d) { if (!v || !*v) return d; return (int)std::strtol(v, nullptr, 10); }
bool asBool(const char* v) { if (!v) return false; char c = v[0]; return c == '1' || c == 't' || c == 'T' || c == 'y' || c == 'Y'; }

// parser.cpp:14-26
Vec3 parseVector3(const std::string& value) {
    std::stringstream ss(value);
    float x, y, z;
    char c1, c2;
    if (!((ss >> x >> c1 >> y >> c2 >> z) && c1 == ',' && c2 == ',')) {
        std::stringstream ss2(value);
        if (!(ss2 >> x >> y >> z)) throw std::runtime_error("Could not parse vector from string: " + value);
    }
    return Vec3(x, y, z);
}
// parser.cpp:28-39
Vec2 parseVector2(const std::string& value) {
    std::stringstream ss(value);
    float x, y;
    char c;
    if (!((ss >> x >> c >> y) && c == ',')) {
        std::stringstream ss2(value);
        if (!(ss2 >> x >> y)) throw std::runtime_error("Could not parse vector from string: " + value);
    }
    return Vec2(x, y);
}

struct Loader {
    std::string baseDir;
    std::unordered_map<std::string, ObjectPtr> refs;
    std::vector<std::shared_ptr<Mesh>> deferred;

    // parser.cpp:41-218
    ObjectPtr parse(const XNode& node) {
        if (node.tag == "ref") {
            const char* id = node.attr("id");
            if (!id || !refs.count(id)) throw std::runtime_error(std::string("No reference found: ") + (id ? id : ""));
            return nullptr;
        }
        PropertyList props;
        std::vector<const XNode*> kids;
        for (const XNode& c : node.kids) {
            std::string nm = c.attr("name") ? c.attr("name") : "";
            const std::string& t = c.tag;
            if (t == "boolean") props.b[nm] = asBool(c.attr("value"));
            else if (t == "integer") props.i[nm] = asInt(c.attr("value"), 0);
            else if (t == "float") props.f[nm] = asFloat(c.attr("value"), 0.f);
            else if (t == "string") props.s[nm] = c.attr("value") ? c.attr("value") : "";
            else if (t == "point") {
                props.p3[nm] = c.attr("value") ? parseVector3(c.attr("value"))
                                               : Vec3(asFloat(c.attr("x"), 0.f), asFloat(c.attr("y"), 0.f), asFloat(c.attr("z"), 0.f));
            } else if (t == "vector2") {
                props.v2[nm] = c.attr("value") ? parseVector2(c.attr("value")) : Vec2(asFloat(c.attr("x"), 0.f), asFloat(c.attr("y"), 0.f));
            } else if (t == "vector" || t == "vector3") {
                props.v3[nm] = c.attr("value") ? parseVector3(c.attr("value"))
                                               : Vec3(asFloat(c.attr("x"), 0.f), asFloat(c.attr("y"), 0.f), asFloat(c.attr("z"), 0.f));
            } else if (t == "color") {
                if (c.attr("value")) { Vec3 v = parseVector3(c.attr("value")); props.c[nm] = Color(v.x, v.y, v.z); }
                else props.c[nm] = Color(asFloat(c.attr("r"), 0.f), asFloat(c.attr("g"), 0.f), asFloat(c.attr("b"), 0.f));
            } else if (t == "transform") {
                Transform tr;
                for (const XNode& st : c.kids) {
                    Transform step;
                    if (st.tag == "translate") {
                        step = Transform::Translate(Vec3(asFloat(st.attr("x"), 0.f), asFloat(st.attr("y"), 0.f), asFloat(st.attr("z"), 0.f)));
                    } else if (st.tag == "scale") {
                        float v = asFloat(st.attr("value"), 0.f);
                        if (v != 0.0f) step = Transform::Scale(v, v, v);
                        else step = Transform::Scale(asFloat(st.attr("x"), 1.f), asFloat(st.attr("y"), 1.f), asFloat(st.attr("z"), 1.f));
                    } else if (st.tag == "rotate") {
                        float ang = asFloat(st.attr("angle"), 0.f);
                        Vec3 axis = st.attr("axis") ? parseVector3(st.attr("axis"))
                                                    : Vec3(asFloat(st.attr("x"), 0.f), asFloat(st.attr("y"), 0.f), asFloat(st.attr("z"), 0.f));
                        step = Transform::Rotate(ang, axis);
                    } else if (st.tag == "lookat") {
                        step = Transform::LookAt(parseVector3(st.attr("origin") ? st.attr("origin") : ""),
                                                 parseVector3(st.attr("target") ? st.attr("target") : ""),
                                                 parseVector3(st.attr("up") ? st.attr("up") : ""));
                    }
                    tr = step * tr;   // parser.cpp:162
                }
                props.t[nm] = tr;
            } else kids.push_back(&c);
        }
        std::string type = node.attr("type") ? node.attr("type") : "";
        if (type.empty()) type = node.tag;
        std::unique_ptr<Object> obj = createInstance(type, props);
        std::string expected = classTypeName(obj->classType());
        if (expected != node.tag && node.tag != "scene")
            throw std::runtime_error("Parsing error: tag <" + node.tag + "> cannot host object of type " + expected);
        if (node.attr("name") && *node.attr("name")) obj->name = node.attr("name");
        ObjectPtr sp(std::move(obj));
        if (node.attr("id") && *node.attr("id")) {
            std::string id = node.attr("id");
            if (refs.count(id)) throw std::runtime_error("Parsing error: id <" + id + "> already exists.");
            refs[id] = sp;
        }
        if (auto mesh = std::dynamic_pointer_cast<Mesh>(sp)) {
            if (!mesh->filename.empty() && std::filesystem::path(mesh->filename).is_relative())
                mesh->filename = (std::filesystem::path(baseDir) / mesh->filename).string();
        }
        sp->setBaseDir(baseDir);
        for (const XNode* k : kids) {
            if (k->tag == "ref") {
                std::string rid = k->attr("id") ? k->attr("id") : "";
                if (!refs.count(rid)) throw std::runtime_error("Parsing error: no object referencing " + rid + " found.");
                sp->addChild(refs[rid]);
            } else if (ObjectPtr c = parse(*k)) {
                sp->addChild(c);
            }
        }
        // Meshes are activated after the whole file is read, in parallel (loading order
        // does not change any result); every other object activates as it is parsed.
        if (auto mesh = std::dynamic_pointer_cast<Mesh>(sp)) deferred.push_back(mesh);
        else if (node.tag != "scene") sp->activate();
        return sp;
    }
};
}  // namespace

// parser.cpp:220-235
std::shared_ptr<Object> loadSceneXML(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("XML parsing failed: cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    std::string src = ss.str();
    XParser xp(src);
    xp.skipMisc();
    XNode root = xp.element();
    Loader ld;
    std::error_code ec;
    auto canon = std::filesystem::canonical(path, ec);
    ld.baseDir = (ec ? std::filesystem::path(path) : canon).parent_path().string();
    ObjectPtr top = ld.parse(root);
    std::atomic<size_t> next{0};
    std::vector<std::string> errors(ld.deferred.size());
    auto work = [&]() {
        for (;;) {
            size_t i = next.fetch_add(1);
            if (i >= ld.deferred.size()) break;
            try { ld.deferred[i]->activate(); } catch (const std::exception& e) { errors[i] = e.what(); }
        }
    };
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    for (auto& e : errors) if (!e.empty()) throw std::runtime_error(e);
    if (root.tag == "scene") top->activate();
    return top;
}

// ---------------------------------------------------------------- OBJ
// mesh.cpp:148-229 for the subset of OBJ the scenes use (v/vt/vn/f, polygons as fans)
void Mesh::loadOBJ(const std::string& fname) {
    std::ifstream f(fname);
    if (!f) throw std::runtime_error("Failed to load OBJ: " + fname);
    std::vector<float> V, T, N;
    struct Idx { int v, t, n; };
    std::vector<Idx> corners;   // three per triangle
    std::string line;
    auto fix = [](int idx, size_t count) { return idx < 0 ? (int)count + idx : idx - 1; };
    while (std::getline(f, line)) {
        const char* p = line.c_str();
        while (*p == ' ' || *p == '\t') ++p;
        if (p[0] == 'v' && (p[1] == ' ' || p[1] == '\t')) {
            char* e; float x = (float)std::strtod(p + 2, &e); float y = (float)std::strtod(e, &e); float z = (float)std::strtod(e, &e);
            V.insert(V.end(), {x, y, z});
        } else if (p[0] == 'v' && p[1] == 't') {
            char* e; float u = (float)std::strtod(p + 2, &e); float v = (float)std::strtod(e, &e);
            T.insert(T.end(), {u, v});
        } else if (p[0] == 'v' && p[1] == 'n') {
            char* e; float x = (float)std::strtod(p + 2, &e); float y = (float)std::strtod(e, &e); float z = (float)std::strtod(e, &e);
            N.insert(N.end(), {x, y, z});
        } else if (p[0] == 'f' && (p[1] == ' ' || p[1] == '\t')) {
            std::vector<Idx> poly;
            std::istringstream is(p + 2);
            std::string tok;
            while (is >> tok) {
                Idx id{-1, -1, -1};
                int a = 0, b = 0, c = 0;
                int nf = 0;
                size_t s1 = tok.find('/');
                a = std::atoi(tok.substr(0, s1).c_str()); nf = 1;
                if (s1 != std::string::npos) {
                    size_t s2 = tok.find('/', s1 + 1);
                    std::string tt = tok.substr(s1 + 1, s2 == std::string::npos ? std::string::npos : s2 - s1 - 1);
                    if (!tt.empty()) { b = std::atoi(tt.c_str()); nf |= 2; }
                    if (s2 != std::string::npos) { c = std::atoi(tok.substr(s2 + 1).c_str()); nf |= 4; }
                }
                id.v = fix(a, V.size() / 3);
                if (nf & 2) id.t = fix(b, T.size() / 2);
                if (nf & 4) id.n = fix(c, N.size() / 3);
                poly.push_back(id);
            }
            for (size_t k = 1; k + 1 < poly.size(); ++k) {
                corners.push_back(poly[0]); corners.push_back(poly[k]); corners.push_back(poly[k + 1]);
            }
        }
    }
    bool hasNormals = !N.empty();
    std::vector<Vec3> gen;
    if (!hasNormals) {
        gen.assign(V.size() / 3, Vec3(0.f));
        for (size_t k = 0; k + 2 < corners.size(); k += 3) {
            auto P = [&](int i) { return Vec3(V[3 * i], V[3 * i + 1], V[3 * i + 2]); };
            Vec3 p0 = P(corners[k].v), p1 = P(corners[k + 1].v), p2 = P(corners[k + 2].v);
            Vec3 wn = Cross(p1 - p0, p2 - p0);
            gen[corners[k].v] = gen[corners[k].v] + wn;
            gen[corners[k + 1].v] = gen[corners[k + 1].v] + wn;
            gen[corners[k + 2].v] = gen[corners[k + 2].v] + wn;
        }
        for (auto& n : gen) { float len = n.length(); if (len > 0.0f) n = n / len; }
    }
    for (const Idx& id : corners) {
        positions.push_back(Vec3(V[3 * id.v], V[3 * id.v + 1], V[3 * id.v + 2]));
        if (hasNormals && id.n >= 0) normals.push_back(Normalize(Vec3(N[3 * id.n], N[3 * id.n + 1], N[3 * id.n + 2])));
        else if (hasNormals) throw std::runtime_error("Mesh: OBJ mixes faces with and without normals: " + fname);
        else normals.push_back(gen[id.v]);
        if (id.t >= 0) uvs.push_back(Vec2(T[2 * id.t], T[2 * id.t + 1]));
        indices.push_back((uint32_t)indices.size());
    }
}

// mesh.cpp:17-28
void Mesh::activate() {
    if (filename.empty()) {
        if (!indices.empty()) { buildAccel(); return; }   // geometry supplied in memory
        throw std::runtime_error("Mesh: filename missing!");
    }
    loadOBJ(filename);
    if (indices.empty()) throw std::runtime_error("Mesh: no geometry loaded!");
    buildAccel();
}

}  // namespace orc
