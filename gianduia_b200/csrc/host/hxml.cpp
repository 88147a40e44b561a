// Scene-file loading: a small XML reader, the reference's element grammar
// (parser.cpp:41-235: property tags, nested objects, <ref id>, transforms composed as
// t = step * t) and the OBJ reader for meshes (mesh.cpp:148-229).
#include <atomic>
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <memory>
#include <fstream>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>

#include "hscene.h"

namespace gndh {

namespace {

struct XmlNode {
    std::string tag;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XmlNode> children;
    const char* attr(const char* k) const {
        for (const auto& a : attrs)
            if (a.first == k) return a.second.c_str();
        return nullptr;
    }
};

class XmlReader {
public:
    explicit XmlReader(const std::string& text) : s_(text) {}
    XmlNode document() {
        skipProlog();
        XmlNode root = element();
        return root;
    }

private:
    const std::string& s_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        // line number of the current offset, for the error message
        size_t line = 1 + std::count(s_.begin(), s_.begin() + std::min(p_, s_.size()), '\n');
        throw std::runtime_error("XML parsing failed: " + what + " (line " + std::to_string(line) + ")");
    }
    bool starts(const char* lit) const { return s_.compare(p_, std::strlen(lit), lit) == 0; }
    void skipSpace() { while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_; }
    void skipUntil(const char* lit) {
        size_t e = s_.find(lit, p_);
        if (e == std::string::npos) fail(std::string("missing '") + lit + "'");
        p_ = e + std::strlen(lit);
    }
    void skipProlog() {
        for (;;) {
            skipSpace();
            if (starts("<?")) skipUntil("?>");
            else if (starts("<!--")) skipUntil("-->");
            else if (starts("<!")) skipUntil(">");
            else return;
        }
    }
    std::string name() {
        size_t b = p_;
        while (p_ < s_.size() && (std::isalnum((unsigned char)s_[p_]) || std::strchr("_-:.", s_[p_]))) ++p_;
        if (b == p_) fail("expected a name");
        return s_.substr(b, p_ - b);
    }
    static std::string decode(const std::string& v) {
        std::string o;
        o.reserve(v.size());
        for (size_t i = 0; i < v.size(); ++i) {
            if (v[i] != '&') { o += v[i]; continue; }
            size_t e = v.find(';', i);
            if (e == std::string::npos) { o += v[i]; continue; }
            std::string ent = v.substr(i + 1, e - i - 1);
            if (ent == "amp") o += '&';
            else if (ent == "lt") o += '<';
            else if (ent == "gt") o += '>';
            else if (ent == "quot") o += '"';
            else if (ent == "apos") o += '\'';
            else o += v.substr(i, e - i + 1);
            i = e;
        }
        return o;
    }
    XmlNode element() {
        if (p_ >= s_.size() || s_[p_] != '<') fail("expected an element");
        ++p_;
        XmlNode n;
        n.tag = name();
        for (;;) {
            skipSpace();
            if (p_ >= s_.size()) fail("unterminated <" + n.tag + ">");
            if (starts("/>")) { p_ += 2; return n; }
            if (s_[p_] == '>') { ++p_; break; }
            std::string k = name();
            skipSpace();
            if (p_ >= s_.size() || s_[p_] != '=') fail("expected '=' after " + k);
            ++p_;
            skipSpace();
            char q = p_ < s_.size() ? s_[p_] : 0;
            if (q != '"' && q != '\'') fail("expected a quoted value for " + k);
            size_t e = s_.find(q, p_ + 1);
            if (e == std::string::npos) fail("unterminated value of " + k);
            n.attrs.emplace_back(k, decode(s_.substr(p_ + 1, e - p_ - 1)));
            p_ = e + 1;
        }
        for (;;) {
            size_t lt = s_.find('<', p_);
            if (lt == std::string::npos) fail("missing </" + n.tag + ">");
            p_ = lt;
            if (starts("<!--")) { skipUntil("-->"); continue; }
            if (starts("<?")) { skipUntil("?>"); continue; }
            if (starts("</")) {
                p_ += 2;
                std::string nm = name();
                if (nm != n.tag) fail("</" + nm + "> closes <" + n.tag + ">");
                skipSpace();
                if (p_ >= s_.size() || s_[p_] != '>') fail("bad closing tag");
                ++p_;
                return n;
            }
            n.children.push_back(element());
        }
    }
};

float toFloat(const char* v, float d) { return (v && *v) ? (float)std::strtod(v, nullptr) : d; }
int toInt(const char* v, int d) { return (v && *v) ? (int)std::strtol(v, nullptr, 10) : d; }
bool toBool(const char* v) { return v && std::strchr("1tTyY", v[0]) && v[0]; }

// parser.cpp:14-39: "x,y,z" with a whitespace-separated fallback
V3 parseV3(const char* value) {
    std::string s = value ? value : "";
    std::stringstream a(s);
    float x, y, z;
    char c1, c2;
    if ((a >> x >> c1 >> y >> c2 >> z) && c1 == ',' && c2 == ',') return gnd::v3(x, y, z);
    std::stringstream b(s);
    if (!(b >> x >> y >> z)) throw std::runtime_error("Could not parse vector from string: " + s);
    return gnd::v3(x, y, z);
}
V2 parseV2(const char* value) {
    std::string s = value ? value : "";
    std::stringstream a(s);
    float x, y;
    char c;
    if ((a >> x >> c >> y) && c == ',') return V2{x, y};
    std::stringstream b(s);
    if (!(b >> x >> y)) throw std::runtime_error("Could not parse vector from string: " + s);
    return V2{x, y};
}

Transform parseTransform(const XmlNode& node) {
    Transform t;
    for (const XmlNode& st : node.children) {
        Transform step;
        if (st.tag == "translate") {
            step = Transform::translate(gnd::v3(toFloat(st.attr("x"), 0.f), toFloat(st.attr("y"), 0.f), toFloat(st.attr("z"), 0.f)));
        } else if (st.tag == "scale") {
            float v = toFloat(st.attr("value"), 0.f);
            if (v != 0.0f) step = Transform::scale(v, v, v);
            else step = Transform::scale(toFloat(st.attr("x"), 1.f), toFloat(st.attr("y"), 1.f), toFloat(st.attr("z"), 1.f));
        } else if (st.tag == "rotate") {
            float angle = toFloat(st.attr("angle"), 0.f);
            V3 axis = st.attr("axis") ? parseV3(st.attr("axis"))
                                      : gnd::v3(toFloat(st.attr("x"), 0.f), toFloat(st.attr("y"), 0.f), toFloat(st.attr("z"), 0.f));
            step = Transform::rotate(angle, axis);
        } else if (st.tag == "lookat") {
            step = Transform::lookAt(parseV3(st.attr("origin")), parseV3(st.attr("target")), parseV3(st.attr("up")));
        }
        t = step * t;
    }
    return t;
}

class Loader {
public:
    explicit Loader(std::string base) : baseDir_(std::move(base)) {}

    std::shared_ptr<GndObject> parse(const XmlNode& node) {
        PropertyList props;
        std::vector<const XmlNode*> kids;
        for (const XmlNode& c : node.children) {
            std::string nm = c.attr("name") ? c.attr("name") : "";
            const std::string& t = c.tag;
            if (t == "boolean") props.setBoolean(nm, toBool(c.attr("value")));
            else if (t == "integer") props.setInteger(nm, toInt(c.attr("value"), 0));
            else if (t == "float") props.setFloat(nm, toFloat(c.attr("value"), 0.f));
            else if (t == "string") props.setString(nm, c.attr("value") ? c.attr("value") : "");
            else if (t == "point") props.setPoint3(nm, c.attr("value") ? parseV3(c.attr("value")) : gnd::v3(toFloat(c.attr("x"), 0.f), toFloat(c.attr("y"), 0.f), toFloat(c.attr("z"), 0.f)));
            else if (t == "vector2") props.setVector2(nm, c.attr("value") ? parseV2(c.attr("value")) : V2{toFloat(c.attr("x"), 0.f), toFloat(c.attr("y"), 0.f)});
            else if (t == "vector" || t == "vector3") props.setVector3(nm, c.attr("value") ? parseV3(c.attr("value")) : gnd::v3(toFloat(c.attr("x"), 0.f), toFloat(c.attr("y"), 0.f), toFloat(c.attr("z"), 0.f)));
            else if (t == "color") props.setColor(nm, c.attr("value") ? parseV3(c.attr("value")) : gnd::v3(toFloat(c.attr("r"), 0.f), toFloat(c.attr("g"), 0.f), toFloat(c.attr("b"), 0.f)));
            else if (t == "transform") props.setTransform(nm, parseTransform(c));
            else kids.push_back(&c);
        }
        std::string type = node.attr("type") ? node.attr("type") : "";
        if (type.empty()) type = node.tag;
        std::unique_ptr<GndObject> obj = GndFactory::getInstance()->createInstance(type, props);
        std::string expected = classTypeToString(obj->getClassType());
        if (expected != node.tag && node.tag != "scene")
            throw std::runtime_error("Parsing error: tag <" + node.tag + "> cannot host object of type " + expected);
        if (node.attr("name") && *node.attr("name")) obj->setName(node.attr("name"));
        std::shared_ptr<GndObject> sp(std::move(obj));
        if (node.attr("id") && *node.attr("id")) {
            std::string id = node.attr("id");
            if (refs_.count(id)) throw std::runtime_error("Parsing error: id <" + id + "> already exists.");
            refs_[id] = sp;
        }
        bool deferred = false;
        if (auto shape = std::dynamic_pointer_cast<ShapeObj>(sp)) {
            if (!shape->filename.empty() && std::filesystem::path(shape->filename).is_relative())
                shape->filename = (std::filesystem::path(baseDir_) / shape->filename).string();
            // mesh files are read later, all at once on every host core (loadPending)
            if (shape->kind == gnd::kShapeMesh && !shape->filename.empty() && shape->positions.empty()) {
                pending_.push_back(shape);
                deferred = true;
            }
        }
        sp->setBaseDir(baseDir_);
        for (const XmlNode* k : kids) {
            if (k->tag == "ref") {
                std::string id = k->attr("id") ? k->attr("id") : "";
                auto it = refs_.find(id);
                if (it == refs_.end()) throw std::runtime_error("Parsing error: no object referencing " + id + " found.");
                sp->addChild(it->second);
            } else {
                sp->addChild(parse(*k));
            }
        }
        if (auto sc = std::dynamic_pointer_cast<Scene>(sp)) {
            sc->deferPreprocess = deferPreprocess;
            sc->deviceBlas = deviceBlas;
            sc->outputPath = outputPath;
            sc->outputName = outputName;
            loadPending();   // the scene's activate builds the mesh trees
        }
        if (!deferred) sp->activate();
        return sp;
    }

    // Reads the deferred mesh files (ShapeObj::activate, mesh.cpp:148-229) on every host
    // core. Parsing does not look at mesh data, so only the loading order changes; the
    // first failing file (in scene-file order) is reported.
    void loadPending() {
        std::vector<std::shared_ptr<ShapeObj>> todo;
        todo.swap(pending_);
        if (todo.empty()) return;
        std::vector<std::exception_ptr> errs(todo.size());
        std::atomic<size_t> next{0};
        auto work = [&]() {
            for (;;) {
                const size_t i = next.fetch_add(1);
                if (i >= todo.size()) break;
                try {
                    todo[i]->activate();
                } catch (...) {
                    errs[i] = std::current_exception();
                }
            }
        };
        const unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)todo.size()));
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t) th.emplace_back(work);
        work();
        for (auto& t : th) t.join();
        for (auto& e : errs)
            if (e) std::rethrow_exception(e);
    }
    bool deferPreprocess = false;
    bool deviceBlas = false;
    std::string outputPath = ".", outputName = "output";

private:
    std::vector<std::shared_ptr<ShapeObj>> pending_;   // mesh shapes whose files are not read yet
    std::string baseDir_;
    std::unordered_map<std::string, std::shared_ptr<GndObject>> refs_;
};

}  // namespace

namespace {
struct ResolverState {
    std::mutex mu;
    std::filesystem::path base = std::filesystem::current_path(), output = std::filesystem::current_path();
    std::string name = "output";   // fileResolver.cpp: the default output name
};
ResolverState& resolver() {
    static ResolverState r;
    return r;
}
}  // namespace

void FileResolver::setBasePath(const std::filesystem::path& p) {
    std::lock_guard<std::mutex> lk(resolver().mu);
    resolver().base = p;
}
void FileResolver::setOutputPath(const std::filesystem::path& p) {
    std::lock_guard<std::mutex> lk(resolver().mu);
    resolver().output = p;
}
void FileResolver::setOutputName(const std::string& n) {
    std::lock_guard<std::mutex> lk(resolver().mu);
    resolver().name = n;
}
std::filesystem::path FileResolver::getBasePath() {
    std::lock_guard<std::mutex> lk(resolver().mu);
    return resolver().base;
}
std::filesystem::path FileResolver::getOutputPath() {
    std::lock_guard<std::mutex> lk(resolver().mu);
    return resolver().output;
}
std::string FileResolver::getOutputName() {
    std::lock_guard<std::mutex> lk(resolver().mu);
    return resolver().name;
}

std::shared_ptr<GndObject> loadFromXML(const std::string& path, bool deferPreprocess, bool deviceBlas) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("XML parsing failed: cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    XmlReader reader(text);
    XmlNode root = reader.document();
    std::error_code ec;
    std::filesystem::path canon = std::filesystem::canonical(path, ec);
    const std::filesystem::path file = ec ? std::filesystem::path(path) : canon;
    // parser.cpp:221-223
    FileResolver::setBasePath(file.parent_path());
    FileResolver::setOutputPath(file.parent_path());
    FileResolver::setOutputName(file.stem().string());
    Loader ld(file.parent_path().string());
    ld.deferPreprocess = deferPreprocess;
    ld.deviceBlas = deviceBlas;
    ld.outputPath = file.parent_path().string();   // parser.cpp:222-223 (FileResolver)
    ld.outputName = file.stem().string();
    auto obj = ld.parse(root);
    ld.loadPending();   // a root that is not a scene
    return obj;
}

// mesh.cpp:148-229 for v / vt / vn / f (polygons split as fans). When the file has no
// normals, smooth normals are generated per original vertex (area-weighted face
// normals, normalised), as the reference does.
namespace {

// strtod(p) converted to float, and the end of the number: std::from_chars takes the plain
// forms; any form it does not parse whole (a sign '+', leading white space other than
// blanks and tabs, hexadecimal, an out-of-range value) goes to strtod itself, so the
// values are strtod's in every case. `lineEnd` is the NUL that ends p's line.
float objFloat(const char* p, const char* lineEnd, const char** end) {
    const char* q = p;
    while (*q == ' ' || *q == '\t') ++q;
    double d;
    const auto r = std::from_chars(q, lineEnd, d);
    if (r.ec == std::errc{} && (r.ptr == lineEnd || *r.ptr == ' ' || *r.ptr == '\t' || *r.ptr == '\r')) {
        *end = r.ptr;
        return (float)d;
    }
    char* e;
    d = std::strtod(p, &e);
    *end = e;
    return (float)d;
}

// strtol(p, 10) and the end of the number, by the same rule.
long objIndex(const char* p, const char* lineEnd, const char** end) {
    long v;
    const auto r = std::from_chars(p, lineEnd, v);
    if (r.ec == std::errc{}) {
        *end = r.ptr;
        return v;
    }
    char* e;
    v = std::strtol(p, &e, 10);
    *end = e;
    return v;
}

}  // namespace

void loadOBJ(const std::string& path, ShapeObj& mesh) {
    // the whole file in one read; each line ends in a NUL where its '\n' was
    std::string text;
    {
        std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "rb"), std::fclose);
        if (!f) throw std::runtime_error("Failed to load OBJ: " + path);
        char buf[1 << 16];
        size_t got;
        while ((got = std::fread(buf, 1, sizeof(buf), f.get())) > 0) text.append(buf, got);
        if (std::ferror(f.get())) throw std::runtime_error("Failed to load OBJ: " + path);
    }
    std::vector<float> V, T, N;
    struct Corner { int v, t, n; };
    std::vector<Corner> corners;
    std::vector<Corner> poly;
    auto resolve = [](long idx, size_t count) -> int { return (int)(idx < 0 ? (long)count + idx : idx - 1); };
    char* const textEnd = text.data() + text.size();
    for (char* line = text.data(); line < textEnd;) {
        char* nl = static_cast<char*>(std::memchr(line, '\n', (size_t)(textEnd - line)));
        char* lineEnd = nl ? nl : textEnd;
        *lineEnd = '\0';   // textEnd is the string's own terminator
        const char* p = line;
        line = lineEnd + 1;
        while (*p == ' ' || *p == '\t') ++p;
        if (p[0] == 'v' && (p[1] == ' ' || p[1] == '\t')) {
            const char* e;
            float x = objFloat(p + 2, lineEnd, &e), y = objFloat(e, lineEnd, &e), z = objFloat(e, lineEnd, &e);
            V.push_back(x); V.push_back(y); V.push_back(z);
        } else if (p[0] == 'v' && p[1] == 't') {
            const char* e;
            float u = objFloat(p + 2, lineEnd, &e), v = objFloat(e, lineEnd, &e);
            T.push_back(u); T.push_back(v);
        } else if (p[0] == 'v' && p[1] == 'n') {
            const char* e;
            float x = objFloat(p + 2, lineEnd, &e), y = objFloat(e, lineEnd, &e), z = objFloat(e, lineEnd, &e);
            N.push_back(x); N.push_back(y); N.push_back(z);
        } else if (p[0] == 'f' && (p[1] == ' ' || p[1] == '\t')) {
            poly.clear();
            const char* q = p + 1;
            for (;;) {
                while (*q == ' ' || *q == '\t') ++q;
                if (!*q || *q == '\r' || *q == '#') break;
                const char* e;
                Corner c{-1, -1, -1};
                c.v = resolve(objIndex(q, lineEnd, &e), V.size() / 3);
                q = e;
                if (*q == '/') {
                    ++q;
                    if (*q != '/') { c.t = resolve(objIndex(q, lineEnd, &e), T.size() / 2); q = e; }
                    if (*q == '/') { ++q; c.n = resolve(objIndex(q, lineEnd, &e), N.size() / 3); q = e; }
                }
                if (c.v < 0 || (size_t)c.v >= V.size() / 3) throw std::runtime_error("OBJ: vertex index out of range in " + path);
                if (c.t >= (int)(T.size() / 2) || c.n >= (int)(N.size() / 3)) throw std::runtime_error("OBJ: attribute index out of range in " + path);
                poly.push_back(c);
                while (*q && *q != ' ' && *q != '\t') ++q;
            }
            for (size_t k = 1; k + 1 < poly.size(); ++k) {
                corners.push_back(poly[0]);
                corners.push_back(poly[k]);
                corners.push_back(poly[k + 1]);
            }
        }
    }
    const bool hasNormals = !N.empty();
    std::vector<V3> gen;
    auto P = [&](int i) { return gnd::v3(V[3 * i], V[3 * i + 1], V[3 * i + 2]); };
    if (!hasNormals) {
        gen.assign(V.size() / 3, gnd::v3s(0.f));
        for (size_t k = 0; k + 2 < corners.size(); k += 3) {
            V3 p0 = P(corners[k].v), p1 = P(corners[k + 1].v), p2 = P(corners[k + 2].v);
            V3 w = gnd::cross(p1 - p0, p2 - p0);
            for (int j = 0; j < 3; ++j) gen[corners[k + j].v] = gen[corners[k + j].v] + w;
        }
        for (V3& n : gen) {
            float len = gnd::length(n);
            if (len > 0.0f) n = gnd::divs(n, len);
        }
    }
    mesh.positions.reserve(corners.size());
    mesh.normals.reserve(corners.size());
    bool anyUV = false, allUV = true;
    for (const Corner& c : corners) {
        if (c.t >= 0) anyUV = true; else allUV = false;
    }
    if (anyUV && !allUV) throw std::runtime_error("OBJ: faces with and without texture coordinates in " + path);
    for (const Corner& c : corners) {
        mesh.positions.push_back(P(c.v));
        if (hasNormals) {
            if (c.n < 0) throw std::runtime_error("OBJ: faces with and without normals in " + path);
            mesh.normals.push_back(gnd::normalize(gnd::v3(N[3 * c.n], N[3 * c.n + 1], N[3 * c.n + 2])));
        } else {
            mesh.normals.push_back(gen[c.v]);
        }
        if (c.t >= 0) mesh.uvs.push_back(V2{T[2 * c.t], T[2 * c.t + 1]});
    }
}

}  // namespace gndh
