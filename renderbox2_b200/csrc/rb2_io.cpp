// Scene files: the reference's XML scene description
// (io/customfilereader.cpp:47-291) and Wavefront OBJ meshes
// (io/objfilereader.cpp:117-216).  Host-only C++; no third-party parser.
#include "rb2_internal.h"
#include "rb2_scene.h"

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>

struct rb2_scene_file {
    std::vector<float> verts;          // 3 per vertex
    std::vector<uint32_t> idx;         // 3 per triangle
    std::vector<uint32_t> tri_mat;     // per triangle
    std::vector<float> albedo, emission;
    std::vector<uint32_t> bsdf;
    std::vector<rb2_material_desc> mats;
    struct Mesh {
        std::string name;
        uint32_t first = 0, count = 0;
    };
    std::vector<Mesh> meshes;
    rb2_scene_file_info info{};
};

namespace {

using rb2::fail;

// ---------------------------------------------------------------- minimal XML
// Elements, text and nesting; attributes are skipped; comments, processing
// instructions, DOCTYPE and CDATA are handled; the five predefined entities
// and numeric character references are decoded.
struct XNode {
    std::string name, text;
    std::vector<XNode> kids;
    const XNode* child(const char* n) const
    {
        for (const XNode& k : kids)
            if (k.name == n) return &k;
        return nullptr;
    }
};

class XmlReader {
public:
    explicit XmlReader(const std::string& s) : s_(s) {}

    bool parse(XNode& root, std::string& err)
    {
        skip_misc();
        if (!element(root, err, 0)) return false;
        skip_misc();
        if (pos_ != s_.size()) return error(err, "content after the root element");
        return true;
    }

private:
    const std::string& s_;
    size_t pos_ = 0;

    bool error(std::string& err, const std::string& what)
    {
        size_t line = 1;
        for (size_t i = 0; i < pos_ && i < s_.size(); i++) line += s_[i] == '\n';
        err = "XML line " + std::to_string(line) + ": " + what;
        return false;
    }
    bool starts(const char* t) const { return s_.compare(pos_, std::strlen(t), t) == 0; }
    void skip_ws()
    {
        while (pos_ < s_.size() && std::isspace((unsigned char)s_[pos_])) pos_++;
    }
    bool skip_until(const char* end)
    {
        const size_t e = s_.find(end, pos_);
        if (e == std::string::npos) return false;
        pos_ = e + std::strlen(end);
        return true;
    }
    // Whitespace, comments, <?...?> and <!DOCTYPE ...> outside elements.
    void skip_misc()
    {
        for (;;) {
            skip_ws();
            if (starts("<!--")) { if (!skip_until("-->")) pos_ = s_.size(); continue; }
            if (starts("<?")) { if (!skip_until("?>")) pos_ = s_.size(); continue; }
            if (starts("<!DOCTYPE")) { if (!skip_until(">")) pos_ = s_.size(); continue; }
            return;
        }
    }
    bool decode(const std::string& raw, std::string& out, std::string& err)
    {
        out.clear();
        for (size_t i = 0; i < raw.size(); i++) {
            if (raw[i] != '&') { out += raw[i]; continue; }
            const size_t e = raw.find(';', i);
            if (e == std::string::npos) return error(err, "unterminated entity");
            const std::string ent = raw.substr(i + 1, e - i - 1);
            if (ent == "lt") out += '<';
            else if (ent == "gt") out += '>';
            else if (ent == "amp") out += '&';
            else if (ent == "quot") out += '"';
            else if (ent == "apos") out += '\'';
            else if (!ent.empty() && ent[0] == '#') {
                const long c = ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X') ? std::strtol(ent.c_str() + 2, nullptr, 16)
                                                                                 : std::strtol(ent.c_str() + 1, nullptr, 10);
                if (c <= 0 || c > 0x7F) return error(err, "non-ASCII character reference");
                out += (char)c;
            } else {
                return error(err, "unknown entity &" + ent + ";");
            }
            i = e;
        }
        return true;
    }
    bool element(XNode& n, std::string& err, int depth)
    {
        if (depth > 256) return error(err, "nesting too deep");
        if (pos_ >= s_.size() || s_[pos_] != '<') return error(err, "expected an element");
        pos_++;
        const size_t b = pos_;
        while (pos_ < s_.size() && !std::isspace((unsigned char)s_[pos_]) && s_[pos_] != '>' && s_[pos_] != '/') pos_++;
        n.name = s_.substr(b, pos_ - b);
        if (n.name.empty()) return error(err, "empty element name");
        // Attributes: skipped, quotes respected.
        while (pos_ < s_.size() && s_[pos_] != '>' && !(s_[pos_] == '/' && pos_ + 1 < s_.size() && s_[pos_ + 1] == '>')) {
            if (s_[pos_] == '"' || s_[pos_] == '\'') {
                const char q = s_[pos_++];
                while (pos_ < s_.size() && s_[pos_] != q) pos_++;
            }
            pos_++;
        }
        if (pos_ >= s_.size()) return error(err, "unterminated start tag <" + n.name + ">");
        if (s_[pos_] == '/') { pos_ += 2; return true; }  // <empty/>
        pos_++;
        std::string raw;
        for (;;) {
            if (pos_ >= s_.size()) return error(err, "missing </" + n.name + ">");
            if (starts("</")) {
                pos_ += 2;
                const size_t e = s_.find('>', pos_);
                if (e == std::string::npos) return error(err, "unterminated end tag");
                std::string close = s_.substr(pos_, e - pos_);
                while (!close.empty() && std::isspace((unsigned char)close.back())) close.pop_back();
                if (close != n.name) return error(err, "</" + close + "> closes <" + n.name + ">");
                pos_ = e + 1;
                break;
            }
            if (starts("<!--")) { if (!skip_until("-->")) return error(err, "unterminated comment"); continue; }
            if (starts("<![CDATA[")) {
                pos_ += 9;
                const size_t e = s_.find("]]>", pos_);
                if (e == std::string::npos) return error(err, "unterminated CDATA");
                raw += s_.substr(pos_, e - pos_);
                pos_ = e + 3;
                continue;
            }
            if (starts("<?")) { if (!skip_until("?>")) return error(err, "unterminated processing instruction"); continue; }
            if (s_[pos_] == '<') {
                n.kids.emplace_back();
                if (!element(n.kids.back(), err, depth + 1)) return false;
                continue;
            }
            raw += s_[pos_++];
        }
        std::string dec;
        if (!decode(raw, dec, err)) return false;
        size_t a = 0, z = dec.size();
        while (a < z && std::isspace((unsigned char)dec[a])) a++;
        while (z > a && std::isspace((unsigned char)dec[z - 1])) z--;
        n.text = dec.substr(a, z - a);
        return true;
    }
};

// "{x, y, z}" / "x y z" / "x,y,z" -> 3 floats (delimiters " {,}", as
// CustomFileReader::get_float3, io/customfilereader.cpp:343-372).
bool parse_float3(const std::string& s, float out[3])
{
    int k = 0;
    size_t i = 0;
    while (k < 3 && i < s.size()) {
        while (i < s.size() && (s[i] == ' ' || s[i] == '{' || s[i] == ',' || s[i] == '}' || s[i] == '\t' || s[i] == '\n' ||
                                s[i] == '\r'))
            i++;
        if (i >= s.size()) break;
        char* end = nullptr;
        errno = 0;
        const float v = std::strtof(s.c_str() + i, &end);
        if (end == s.c_str() + i) return false;
        out[k++] = v;
        i = (size_t)(end - s.c_str());
    }
    return k == 3;
}

std::string dir_of(const std::string& path)
{
    const size_t p = path.find_last_of('/');
    return p == std::string::npos ? std::string() : path.substr(0, p + 1);
}

bool ends_with(const std::string& s, const char* suf)
{
    const size_t n = std::strlen(suf);
    if (s.size() < n) return false;
    for (size_t i = 0; i < n; i++)
        if (std::tolower((unsigned char)s[s.size() - n + i]) != suf[i]) return false;
    return true;
}

// ------------------------------------------------------------------------ OBJ
// Triangles go to the mesh of the last "o" line; a face of n vertices gives
// n - 2 triangles (fan from its first vertex).  Only the position index of
// each face vertex is used (v, v/vt, v//vn, v/vt/vn).
int load_obj(const std::string& path, rb2_scene_file& f)
{
    std::ifstream in(path);
    if (!in) return fail(RB2_EIO, "cannot open " + path);
    std::string line;
    uint64_t lineno = 0;
    auto bad = [&](const std::string& what) { return fail(RB2_EFORMAT, path + ":" + std::to_string(lineno) + ": " + what); };
    auto cur_mesh = [&]() -> rb2_scene_file::Mesh& {
        if (f.meshes.empty()) {
            f.meshes.push_back({});
            f.meshes.back().name = "default";
            f.meshes.back().first = (uint32_t)(f.idx.size() / 3);
        }
        return f.meshes.back();
    };
    std::vector<long> face;
    while (std::getline(in, line)) {
        lineno++;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        std::istringstream ls(line);
        std::string tag;
        if (!(ls >> tag)) continue;
        if (tag == "o") {
            std::string name;
            std::getline(ls >> std::ws, name);
            while (!name.empty() && std::isspace((unsigned char)name.back())) name.pop_back();
            f.meshes.push_back({});
            f.meshes.back().name = name;
            f.meshes.back().first = (uint32_t)(f.idx.size() / 3);
        } else if (tag == "v") {
            float x, y, z;
            if (!(ls >> x >> y >> z)) return bad("vertex needs three coordinates");
            f.verts.insert(f.verts.end(), {x, y, z});
            if (f.verts.size() / 3 > 0xFFFFFFFEull) return bad("too many vertices");
        } else if (tag == "f") {
            face.clear();
            std::string tok;
            const long nv = (long)(f.verts.size() / 3);
            while (ls >> tok) {
                char* end = nullptr;
                const long v = std::strtol(tok.c_str(), &end, 10);
                if (end == tok.c_str() || (*end != '\0' && *end != '/')) return bad("bad face vertex '" + tok + "'");
                const long a = v > 0 ? v - 1 : nv + v;  // 1-based, or relative when negative
                if (v == 0 || a < 0 || a >= nv) return bad("face index out of range");
                face.push_back(a);
            }
            if (face.size() < 3) return bad("face with fewer than three vertices");
            rb2_scene_file::Mesh& m = cur_mesh();
            for (size_t k = 1; k + 1 < face.size(); k++) {
                f.idx.insert(f.idx.end(), {(uint32_t)face[0], (uint32_t)face[k], (uint32_t)face[k + 1]});
                m.count++;
            }
        }
        // vn, vt, g, s, usemtl, mtllib and others carry nothing the path uses.
    }
    if (f.idx.empty()) return fail(RB2_EFORMAT, path + ": no faces");
    return RB2_OK;
}

rb2_material_desc default_material()
{
    rb2_material_desc d{};
    d.n_layers = 1;
    d.layer[0].type = RB2_BSDF_LAMBERTIAN;
    d.layer[0].color[0] = d.layer[0].color[1] = d.layer[0].color[2] = 0.5f;
    return d;
}

int bsdf_code(const std::string& t)
{
    if (t == "lambertian") return RB2_BSDF_LAMBERTIAN;
    if (t == "orennayar") return RB2_BSDF_OREN_NAYAR;
    if (t == "mirror") return RB2_BSDF_MIRROR;
    if (t == "glass") return RB2_BSDF_GLASS;
    if (t == "microfacet") return RB2_BSDF_MICROFACET;
    return -1;
}

int load_xml(const std::string& path, rb2_scene_file& f)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) return fail(RB2_EIO, "cannot open " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string text = ss.str();
    XNode root;
    std::string err;
    if (!XmlReader(text).parse(root, err)) return fail(RB2_EFORMAT, path + ": " + err);
    if (root.name != "scene") return fail(RB2_EFORMAT, path + ": root element is not <scene>");
    const XNode* files = root.child("files");
    const XNode* file = files ? files->child("file") : nullptr;
    if (!file || file->text.empty()) return fail(RB2_EFORMAT, path + ": <files><file> missing");
    if (const XNode* count = files->child("count"))
        if (std::atoi(count->text.c_str()) != 1) return fail(RB2_ENOTSUP, path + ": exactly one OBJ file is supported");
    int rc = load_obj(dir_of(path) + file->text, f);
    if (rc) return rc;

    std::map<std::string, uint32_t> mat_of;
    for (const XNode& m : root.kids) {
        if (m.name != "material") continue;
        const XNode* name = m.child("name");
        const XNode* bsdf = m.child("bsdf");
        if (!name || !bsdf) return fail(RB2_EFORMAT, path + ": material without <name> or <bsdf>");
        rb2_material_desc desc{};
        for (const XNode& bx : bsdf->kids) {
            if (bx.name != "bxdf") continue;
            if (desc.n_layers == 4) return fail(RB2_EFORMAT, path + ": more than 4 layers in material " + name->text);
            rb2_bsdf_layer& L = desc.layer[desc.n_layers++];
            const XNode* type = bx.child("type");
            const int code = type ? bsdf_code(type->text) : -1;
            if (code < 0) return fail(RB2_EFORMAT, path + ": unknown bxdf type in material " + name->text);
            L.type = (uint32_t)code;
            L.color[0] = L.color[1] = L.color[2] = 0.5f;
            auto num = [&](const char* tag, float& out) -> bool {
                const XNode* e = bx.child(tag);
                if (!e) return false;
                char* end = nullptr;
                out = std::strtof(e->text.c_str(), &end);
                return end != e->text.c_str();
            };
            auto vec = [&](const char* tag, float* out) -> bool {
                const XNode* e = bx.child(tag);
                return e && parse_float3(e->text, out);
            };
            if (const XNode* refl = bx.child("reflectance"))
                if (!parse_float3(refl->text, L.color))
                    return fail(RB2_EFORMAT, path + ": bad reflectance in " + name->text);
            const std::string where = path + ": material " + name->text + ": ";
            if (code == RB2_BSDF_OREN_NAYAR && !num("sigma", L.sigma_deg)) return fail(RB2_EFORMAT, where + "<sigma> missing");
            if (code == RB2_BSDF_GLASS && !(num("etai", L.etai) && num("etat", L.etat)))
                return fail(RB2_EFORMAT, where + "glass needs <etai> and <etat>");
            if (code == RB2_BSDF_MICROFACET) {
                const XNode* dist = bx.child("distribution");
                if (!dist || dist->text != "blinn") return fail(RB2_EFORMAT, where + "only the blinn distribution exists");
                if (!num("exponent", L.exponent)) return fail(RB2_EFORMAT, where + "<exponent> missing");
                const XNode* ft = bx.child("fresnel_type");
                const std::string fts = ft ? ft->text : std::string("fresnel_noop");
                if (fts == "fresnel_conductor") {
                    L.fresnel = RB2_FRESNEL_CONDUCTOR;
                    if (!(vec("eta", L.eta) && vec("k", L.k))) return fail(RB2_EFORMAT, where + "conductor needs <eta> and <k>");
                } else if (fts == "fresnel_dielectric") {
                    L.fresnel = RB2_FRESNEL_DIELECTRIC;
                    if (!(num("etai", L.etai) && num("etat", L.etat)))
                        return fail(RB2_EFORMAT, where + "dielectric needs <etai> and <etat>");
                } else if (fts == "fresnel_noop") {
                    L.fresnel = RB2_FRESNEL_NOOP;
                } else {
                    return fail(RB2_EFORMAT, where + "unknown fresnel_type " + fts);
                }
            }
        }
        if (desc.n_layers == 0) return fail(RB2_EFORMAT, path + ": material " + name->text + " has no <bxdf>");
        mat_of[name->text] = (uint32_t)f.bsdf.size();
        f.bsdf.push_back(desc.layer[0].type);
        f.albedo.insert(f.albedo.end(), desc.layer[0].color, desc.layer[0].color + 3);
        f.emission.insert(f.emission.end(), {0.0f, 0.0f, 0.0f});
        f.mats.push_back(desc);
    }
    std::vector<uint32_t> mesh_mat(f.meshes.size(), 0u);
    for (const XNode& o : root.kids) {
        if (o.name != "object") continue;
        const XNode* name = o.child("name");
        const XNode* mat = o.child("material");
        if (!name || !mat) return fail(RB2_EFORMAT, path + ": <object> without <name> or <material>");
        auto it = mat_of.find(mat->text);
        if (it == mat_of.end()) return fail(RB2_EFORMAT, path + ": object " + name->text + " names unknown material");
        for (size_t i = 0; i < f.meshes.size(); i++)
            if (f.meshes[i].name == name->text) { mesh_mat[i] = it->second; break; }
    }
    if (const XNode* lights = root.child("lightobjects")) {
        for (const XNode& l : lights->kids) {
            if (l.name != "light") continue;
            const XNode* name = l.child("name");
            const XNode* le = l.child("Le");
            float rgb[3];
            if (!name || !le || !parse_float3(le->text, rgb)) return fail(RB2_EFORMAT, path + ": bad <light>");
            const uint32_t id = (uint32_t)f.bsdf.size();
            f.bsdf.push_back(RB2_BSDF_EMITTER);
            f.mats.push_back(rb2_material_desc{});
            f.albedo.insert(f.albedo.end(), {0.0f, 0.0f, 0.0f});
            f.emission.insert(f.emission.end(), rgb, rgb + 3);
            for (size_t i = 0; i < f.meshes.size(); i++)
                if (f.meshes[i].name == name->text) { mesh_mat[i] = id; break; }
        }
    }
    if (f.bsdf.empty()) {  // no materials declared: one default Lambertian
        f.bsdf.push_back(RB2_BSDF_LAMBERTIAN);
        f.albedo.insert(f.albedo.end(), {0.5f, 0.5f, 0.5f});
        f.emission.insert(f.emission.end(), {0.0f, 0.0f, 0.0f});
        f.mats.push_back(default_material());
    }
    f.tri_mat.assign(f.idx.size() / 3, 0u);
    for (size_t i = 0; i < f.meshes.size(); i++)
        for (uint32_t t = 0; t < f.meshes[i].count; t++) f.tri_mat[f.meshes[i].first + t] = mesh_mat[i];
    if (const XNode* cam = root.child("camera")) {
        const XNode* e = cam->child("position");
        const XNode* l = cam->child("lookat");
        const XNode* u = cam->child("up");
        if (e && l && u && parse_float3(e->text, f.info.eye) && parse_float3(l->text, f.info.lookat) &&
            parse_float3(u->text, f.info.up)) {
            f.info.has_camera = 1;
            f.info.fov_deg = 90.0f;
            if (const XNode* fov = cam->child("fov")) {
                char* end = nullptr;
                const float v = std::strtof(fov->text.c_str(), &end);
                if (end != fov->text.c_str() && v > 0.0f && v < 180.0f) f.info.fov_deg = v;
            }
        }
    }
    return RB2_OK;
}

}  // namespace

extern "C" {

int rb2_scene_file_load(const char* path, rb2_scene_file** out)
{
    if (!path || !out) return fail(RB2_EINVAL, "null argument");
    *out = nullptr;
    std::unique_ptr<rb2_scene_file> f(new rb2_scene_file());
    const std::string p(path);
    int rc;
    if (ends_with(p, ".obj")) {
        rc = load_obj(p, *f);
        if (!rc) {
            f->bsdf.assign(1, RB2_BSDF_LAMBERTIAN);
            f->albedo = {0.5f, 0.5f, 0.5f};
            f->emission = {0.0f, 0.0f, 0.0f};
            f->mats.assign(1, default_material());
            f->tri_mat.assign(f->idx.size() / 3, 0u);
        }
    } else {
        rc = load_xml(p, *f);
    }
    if (rc) return rc;
    rb2_scene_file_info& i = f->info;
    i.n_vertices = (uint32_t)(f->verts.size() / 3);
    i.n_triangles = (uint32_t)(f->idx.size() / 3);
    i.n_materials = (uint32_t)f->bsdf.size();
    i.n_meshes = (uint32_t)f->meshes.size();
    i.n_lights = 0;
    for (uint32_t m : f->tri_mat) i.n_lights += f->bsdf[m] == RB2_BSDF_EMITTER ? 1u : 0u;  // emissive triangles
    *out = f.release();
    return RB2_OK;
}

int rb2_scene_file_info_get(const rb2_scene_file* f, rb2_scene_file_info* out)
{
    if (!f || !out) return fail(RB2_EINVAL, "null argument");
    *out = f->info;
    return RB2_OK;
}

const float* rb2_scene_file_vertices(const rb2_scene_file* f) { return f ? f->verts.data() : nullptr; }
const uint32_t* rb2_scene_file_indices(const rb2_scene_file* f) { return f ? f->idx.data() : nullptr; }
const uint32_t* rb2_scene_file_tri_material(const rb2_scene_file* f) { return f ? f->tri_mat.data() : nullptr; }
const float* rb2_scene_file_albedo(const rb2_scene_file* f) { return f ? f->albedo.data() : nullptr; }
const float* rb2_scene_file_emission(const rb2_scene_file* f) { return f ? f->emission.data() : nullptr; }
const uint32_t* rb2_scene_file_bsdf_types(const rb2_scene_file* f) { return f ? f->bsdf.data() : nullptr; }
const rb2_material_desc* rb2_scene_file_materials(const rb2_scene_file* f) { return f ? f->mats.data() : nullptr; }

int rb2_scene_file_mesh(const rb2_scene_file* f, uint32_t i, const char** name, uint32_t* first, uint32_t* count)
{
    if (!f || !name || !first || !count) return fail(RB2_EINVAL, "null argument");
    if (i >= f->meshes.size()) return fail(RB2_EINVAL, "mesh index out of range");
    *name = f->meshes[i].name.c_str();
    *first = f->meshes[i].first;
    *count = f->meshes[i].count;
    return RB2_OK;
}

void rb2_scene_file_free(rb2_scene_file* f) { delete f; }

}  // extern "C"
