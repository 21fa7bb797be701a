// scene_file.cu — Aurora's scene file (the JSON schema read by JsonParser,
// Aurora/src/translator/jsonParser.cpp:30-661) flattened on the host into the
// camera-space arrays of aur_scene_desc, the way Renderer::buildRenderEnvironment
// (renderer.cpp:99-145) lays them out: geometry objects first (attribute i =
// object i), then the light shapes (attribute nobj + j, constant material,
// emission = color * 2^exposure).
//
//   options    resolution, pixelsamples, lightsamples, mindepth, maxdepth, filename
//   renderCam  fov (slope factor, camera.cpp:51-52), transforms (camera to world)
//   shaders    texture2DShader, triplanarTextureShader (texture files in OpenEXR: scanline,
//              NONE / RLE / ZIPS / ZIP; or PFM)
//   materials  matteMaterial, kelemenMaterial, metalMaterial, glassMaterial; normalmap
//   objects    geometry (OBJ triangles, optional Loop subdivision), light (square), envlight
//
// Objects of a JSON object are visited in key order, as the reference's JSON
// library (an ordered map) visits them, so global triangle ids and attribute
// indices follow the reference's append order. Transforms use the reference's
// FP32 matrix arithmetic (core/transform.cpp:36-136, core/matrix4x4.cpp:49-150).
#include "aur_capi_internal.h"
#include "aur_host_math.h"
#include "aur_image_io.h"
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

struct aur_scene_file {
    std::vector<float> verts, corner_normals, corner_uvs, attr_emission, texels;
    std::vector<float> tex_scale;   // per texture: 0 = texture2DShader, > 0 = triplanar scale
    std::vector<float> attr_c2o;    // per attribute: cameraToObject, 16 floats
    std::vector<uint32_t> tri_vidx;
    std::vector<int32_t> tri_attr, attr_material, tex_dims;
    std::vector<aur_material_desc> materials;
    std::vector<aur_light_desc> lights;
    float fov = 1.f;
    int32_t width = 0, height = 0;
    aur_render_opts opts{};
    int32_t light_samples = 1;
    std::string output;
};

namespace aur {
namespace {

// ------------------------------------------------------------------ JSON
struct JValue {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<JValue> arr;
    std::map<std::string, JValue> obj;   // visited in key order
    const JValue* get(const char* k) const {
        if (kind != Obj) return nullptr;
        auto it = obj.find(k);
        return it == obj.end() ? nullptr : &it->second;
    }
};

struct JParser {
    const char* p;
    const char* end;
    const char* begin;
    std::string err;

    int line_of(const char* q) const {
        int l = 1;
        for (const char* c = begin; c < q && c < end; ++c) l += *c == '\n';
        return l;
    }
    bool fail(const char* what) {
        if (err.empty()) err = std::string(what) + " at line " + std::to_string(line_of(p));
        return false;
    }
    void ws() {
        while (p < end) {
            if (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r') ++p;
            else if (*p == '/' && p + 1 < end && p[1] == '/') { while (p < end && *p != '\n') ++p; }
            else if (*p == '/' && p + 1 < end && p[1] == '*') {
                p += 2;
                while (p + 1 < end && !(p[0] == '*' && p[1] == '/')) ++p;
                p = p + 2 <= end ? p + 2 : end;
            } else break;
        }
    }
    bool lit(const char* s) {
        const size_t n = strlen(s);
        if ((size_t)(end - p) < n || strncmp(p, s, n) != 0) return false;
        p += n;
        return true;
    }
    static void put_utf8(std::string& s, unsigned cp) {
        if (cp < 0x80) s += (char)cp;
        else if (cp < 0x800) { s += (char)(0xC0 | (cp >> 6)); s += (char)(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000) {
            s += (char)(0xE0 | (cp >> 12)); s += (char)(0x80 | ((cp >> 6) & 0x3F)); s += (char)(0x80 | (cp & 0x3F));
        } else {
            s += (char)(0xF0 | (cp >> 18)); s += (char)(0x80 | ((cp >> 12) & 0x3F));
            s += (char)(0x80 | ((cp >> 6) & 0x3F)); s += (char)(0x80 | (cp & 0x3F));
        }
    }
    bool hex4(unsigned* v) {
        if (end - p < 4) return fail("truncated \\u escape");
        *v = 0;
        for (int i = 0; i < 4; ++i, ++p) {
            const char c = *p;
            *v <<= 4;
            if (c >= '0' && c <= '9') *v |= (unsigned)(c - '0');
            else if (c >= 'a' && c <= 'f') *v |= (unsigned)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') *v |= (unsigned)(c - 'A' + 10);
            else return fail("bad \\u escape");
        }
        return true;
    }
    bool string(std::string& out) {
        ++p;   // opening quote
        out.clear();
        while (p < end && *p != '"') {
            if (*p == '\\') {
                if (++p >= end) return fail("truncated escape");
                switch (*p) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        ++p;
                        unsigned cp;
                        if (!hex4(&cp)) return false;
                        if (cp >= 0xD800 && cp < 0xDC00 && end - p >= 6 && p[0] == '\\' && p[1] == 'u') {
                            p += 2;
                            unsigned lo;
                            if (!hex4(&lo)) return false;
                            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                        }
                        put_utf8(out, cp);
                        continue;
                    }
                    default: return fail("bad escape");
                }
                ++p;
            } else {
                out += *p++;
            }
        }
        if (p >= end) return fail("unterminated string");
        ++p;
        return true;
    }
    bool value(JValue& v, int depth) {
        if (depth > 256) return fail("nesting too deep");
        ws();
        if (p >= end) return fail("unexpected end of file");
        if (*p == '{') {
            v.kind = JValue::Obj;
            ++p;
            ws();
            if (p < end && *p == '}') { ++p; return true; }
            while (true) {
                ws();
                if (p >= end || *p != '"') return fail("expected a key");
                std::string key;
                if (!string(key)) return false;
                ws();
                if (p >= end || *p != ':') return fail("expected ':'");
                ++p;
                JValue child;
                if (!value(child, depth + 1)) return false;
                v.obj[key] = std::move(child);   // a repeated key keeps the last value
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == '}') { ++p; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (*p == '[') {
            v.kind = JValue::Arr;
            ++p;
            ws();
            if (p < end && *p == ']') { ++p; return true; }
            while (true) {
                JValue child;
                if (!value(child, depth + 1)) return false;
                v.arr.push_back(std::move(child));
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == ']') { ++p; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (*p == '"') { v.kind = JValue::Str; return string(v.str); }
        if (lit("true")) { v.kind = JValue::Bool; v.b = true; return true; }
        if (lit("false")) { v.kind = JValue::Bool; v.b = false; return true; }
        if (lit("null")) { v.kind = JValue::Null; return true; }
        if (*p == '-' || (*p >= '0' && *p <= '9')) {
            std::string tok;
            while (p < end && (strchr("+-.eE", *p) || (*p >= '0' && *p <= '9'))) tok += *p++;
            char* e = nullptr;
            errno = 0;
            v.num = strtod(tok.c_str(), &e);
            if (!e || *e != '\0') return fail("bad number");
            v.kind = JValue::Num;
            return true;
        }
        return fail("unexpected character");
    }
};

// ------------------------------------------------------------------ errors
struct LoadError {
    aur_status status;
    std::string msg;
};
[[noreturn]] void throw_load(aur_status s, const std::string& m) { throw LoadError{s, m}; }

const JValue& need(const JValue& o, const char* key, const std::string& where) {
    const JValue* v = o.get(key);
    if (!v) throw_load(AUR_ERR_PARSE, where + ": missing \"" + key + "\"");
    return *v;
}
double need_num(const JValue& o, const char* key, const std::string& where) {
    const JValue& v = need(o, key, where);
    if (v.kind == JValue::Num) return v.num;
    if (v.kind == JValue::Bool) return v.b ? 1.0 : 0.0;
    throw_load(AUR_ERR_PARSE, where + ": \"" + key + "\" is not a number");
}
std::string need_str(const JValue& o, const char* key, const std::string& where) {
    const JValue& v = need(o, key, where);
    if (v.kind != JValue::Str) throw_load(AUR_ERR_PARSE, where + ": \"" + key + "\" is not a string");
    return v.str;
}
void need_nums(const JValue& o, const char* key, int n, double* out, const std::string& where) {
    const JValue& v = need(o, key, where);
    if (v.kind != JValue::Arr || (int)v.arr.size() != n)
        throw_load(AUR_ERR_PARSE, where + ": \"" + key + "\" must be an array of " + std::to_string(n) + " numbers");
    for (int i = 0; i < n; ++i) {
        if (v.arr[i].kind != JValue::Num) throw_load(AUR_ERR_PARSE, where + ": \"" + key + "\" holds a non-number");
        out[i] = v.arr[i].num;
    }
}

// ------------------------------------------------------------------ Transform (FP32, as the reference)
struct M4 { float m[4][4]; };

M4 identity() {
    M4 r{};
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.f;
    return r;
}
M4 mul(const M4& a, const M4& b) {        // Matrix4x4::operator* (matrix4x4.cpp:49-60)
    M4 r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j] + a.m[i][3] * b.m[3][j];
    return r;
}
bool inverse(const M4& in, M4* out) { return invert4_gj(&in.m[0][0], &out->m[0][0]); }

struct Xform {
    M4 m = identity(), inv = identity();
    void post(const M4& t) {               // m *= t; mInv = m.inverse() (transform.cpp:43-104)
        m = mul(m, t);
        if (!inverse(m, &inv)) throw_load(AUR_ERR_PARSE, "singular transform");
    }
    Xform operator*(const Xform& b) const { // Transform::operator* (transform.cpp:186-191)
        Xform r;
        r.m = mul(m, b.m);
        r.inv = mul(b.inv, inv);
        return r;
    }
    Xform inverted() const { Xform r; r.m = inv; r.inv = m; return r; }
    float3 point(float3 p) const {         // Transform::operator()(Point) (transform.cpp:203-211)
        const float xp = m.m[0][0] * p.x + m.m[0][1] * p.y + m.m[0][2] * p.z + m.m[0][3];
        const float yp = m.m[1][0] * p.x + m.m[1][1] * p.y + m.m[1][2] * p.z + m.m[1][3];
        const float zp = m.m[2][0] * p.x + m.m[2][1] * p.y + m.m[2][2] * p.z + m.m[2][3];
        const float wp = m.m[3][0] * p.x + m.m[3][1] * p.y + m.m[3][2] * p.z + m.m[3][3];
        if (wp == 1.f) return make_float3(xp, yp, zp);
        const float iw = 1.f / wp;          // Point::operator/ multiplies by the reciprocal
        return make_float3(xp * iw, yp * iw, zp * iw);
    }
    float3 vector(float3 v) const {        // Transform::operator()(Vector) (transform.cpp:222-228)
        return make_float3(m.m[0][0] * v.x + m.m[0][1] * v.y + m.m[0][2] * v.z,
                           m.m[1][0] * v.x + m.m[1][1] * v.y + m.m[1][2] * v.z,
                           m.m[2][0] * v.x + m.m[2][1] * v.y + m.m[2][2] * v.z);
    }
};

M4 mat(float a, float b, float c, float d, float e, float f, float g, float h, float i, float j, float k, float l) {
    M4 r{};
    const float v[12] = {a, b, c, d, e, f, g, h, i, j, k, l};
    for (int q = 0; q < 12; ++q) r.m[q / 4][q % 4] = v[q];
    r.m[3][3] = 1.f;
    return r;
}
float radians_f(float deg) { return (float)(deg * M_PI / 180.f); }   // math_utils.h:211-214

// getTransformAttr (jsonParser.cpp:163-222): a list of single-key objects applied in order
Xform parse_transforms(const JValue* list, const std::string& where) {
    Xform t;
    if (!list) throw_load(AUR_ERR_PARSE, where + ": missing \"transforms\"");
    if (list->kind == JValue::Obj && list->obj.empty()) return t;   // PyAurora writes an empty list as {}
    if (list->kind != JValue::Arr) throw_load(AUR_ERR_PARSE, where + ": \"transforms\" must be an array");
    for (const JValue& op : list->arr) {
        if (op.kind != JValue::Obj || op.obj.empty()) throw_load(AUR_ERR_PARSE, where + ": bad transform entry");
        const std::string& key = op.obj.begin()->first;
        const JValue& v = op.obj.begin()->second;
        if (key == "translate" || key == "scale") {
            double n[3];
            if (v.kind != JValue::Arr || v.arr.size() != 3) throw_load(AUR_ERR_PARSE, where + ": " + key + " needs 3 numbers");
            for (int i = 0; i < 3; ++i) {
                if (v.arr[i].kind != JValue::Num) throw_load(AUR_ERR_PARSE, where + ": " + key + " needs 3 numbers");
                n[i] = v.arr[i].num;
            }
            const float x = (float)n[0], y = (float)n[1], z = (float)n[2];
            if (key == "translate") t.post(mat(1, 0, 0, x, 0, 1, 0, y, 0, 0, 1, z));
            else t.post(mat(x, 0, 0, 0, 0, y, 0, 0, 0, 0, z, 0));
        } else if (key == "rotateX" || key == "rotateY" || key == "rotateZ") {
            if (v.kind != JValue::Num) throw_load(AUR_ERR_PARSE, where + ": " + key + " needs a number");
            const float a = radians_f((float)v.num);
            const float s = sinf(a), c = cosf(a);
            if (key == "rotateX") t.post(mat(1, 0, 0, 0, 0, c, -s, 0, 0, s, c, 0));
            else if (key == "rotateY") t.post(mat(c, 0, s, 0, 0, 1, 0, 0, -s, 0, c, 0));
            else t.post(mat(c, -s, 0, 0, s, c, 0, 0, 0, 0, 1, 0));
        }
        // other keys are ignored, as the reference ignores them
    }
    return t;
}

// ------------------------------------------------------------------ float3 helpers (FP32)
float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
float3 scl(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
float3 crs(float3 a, float3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
float3 nrm(float3 v) {                       // Vector::length / operator/ (vector.h:65-80)
    float l = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    if (l == 0.f) l = 0.0001f;
    const float inv = 1.f / l;
    return f3(v.x * inv, v.y * inv, v.z * inv);
}

// ------------------------------------------------------------------ OBJ (objParser.cpp, objTriangleMesh.cpp:26-92)
struct Corners {                      // one entry per triangle corner, object space
    std::vector<float3> P, N;
    std::vector<float2> UV;
    bool has_uv = false;
};

int obj_index(const std::string& tok, int field) {   // field 0: vertex, 1: uv, 2: normal; 0 when absent
    int f = 0;
    size_t start = 0;
    for (size_t i = 0; i <= tok.size(); ++i) {
        if (i == tok.size() || tok[i] == '/') {
            if (f == field) return i > start ? atoi(tok.substr(start, i - start).c_str()) : 0;
            ++f;
            start = i + 1;
        }
    }
    return 0;
}

Corners read_obj(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw_load(AUR_ERR_IO, "cannot open OBJ file " + path);
    std::vector<float3> pts, nrms;
    std::vector<float2> uvs;
    std::vector<int> vi, ti, ni;
    std::string line;
    int lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        std::istringstream ss(line);
        std::string op;
        ss >> op;
        if (op == "v") {
            float x = 0, y = 0, z = 0;
            ss >> x >> y >> z;
            pts.push_back(f3(x, y, z));
        } else if (op == "vn") {
            float x = 0, y = 0, z = 0;
            ss >> x >> y >> z;
            nrms.push_back(f3(x, y, z));
        } else if (op == "vt") {
            float u = 0, v = 0;
            ss >> u >> v;
            uvs.push_back(make_float2(u, v));
        } else if (op == "f") {
            std::string c[4];
            ss >> c[0] >> c[1] >> c[2] >> c[3];
            if (c[2].empty()) throw_load(AUR_ERR_PARSE, path + ":" + std::to_string(lineno) + ": face with fewer than 3 corners");
            if (!c[3].empty())
                throw_load(AUR_ERR_PARSE, path + ":" + std::to_string(lineno) + ": only triangles are read (as the reference)");
            for (int k = 0; k < 3; ++k) {
                vi.push_back(obj_index(c[k], 0));
                ti.push_back(obj_index(c[k], 1));
                ni.push_back(obj_index(c[k], 2));
            }
        }
    }
    Corners cs;
    const size_t n = vi.size();
    cs.P.resize(n);
    cs.N.resize(n);
    cs.has_uv = !uvs.empty();
    if (cs.has_uv) cs.UV.resize(n);
    for (size_t i = 0; i < n; ++i) {
        if (vi[i] < 1 || (size_t)vi[i] > pts.size()) throw_load(AUR_ERR_PARSE, path + ": vertex index out of range");
        cs.P[i] = pts[vi[i] - 1];
        if (ni[i] >= 1 && (size_t)ni[i] <= nrms.size()) {
            cs.N[i] = nrms[ni[i] - 1];
            if (cs.N[i].x == 0.f && cs.N[i].y == 0.f && cs.N[i].z == 0.f) cs.N[i] = f3(0, 1, 0);   // as the reference
        } else {
            cs.N[i] = f3(0, 0, 0);   // filled with the face normal below
        }
        if (cs.has_uv) {
            if (ti[i] < 1 || (size_t)ti[i] > uvs.size()) throw_load(AUR_ERR_PARSE, path + ": uv index out of range");
            cs.UV[i] = uvs[ti[i] - 1];
        }
    }
    // Extension: corners without a normal take the triangle's geometric normal (the
    // reference requires a normal on every corner).
    for (size_t t = 0; t + 2 < n; t += 3)
        for (int k = 0; k < 3; ++k)
            if (cs.N[t + k].x == 0.f && cs.N[t + k].y == 0.f && cs.N[t + k].z == 0.f)
                cs.N[t + k] = nrm(crs(sub(cs.P[t + 1], cs.P[t]), sub(cs.P[t + 2], cs.P[t])));
    return cs;
}

// ------------------------------------------------------------------ Loop subdivision
// Loop's scheme (C. Loop, "Smooth Subdivision Surfaces Based on Triangles", 1987) in the
// form of LoopSubdivMesh (loopSubdivMesh.cpp:167-744): vertices are welded by exact
// position; even vertices take (1 - n beta) P + beta * ring (beta = 3/16 at valence 3,
// else 3/(8n)), boundary ones 3/4 P + 1/8 (both boundary neighbours); odd vertices
// 3/8 (edge ends) + 1/8 (opposite vertices), boundary 1/2 (edge ends). After the last
// level every vertex moves to its limit position (gamma = 1/(n + 3/(8 beta)); boundary
// 3/5 P + 1/5 neighbours) and takes the limit normal cross(T, S) of its ring. UVs are
// per corner and interpolated with the same weights unless they differ across an
// edge or around a vertex (a seam), where they interpolate linearly / stay.
struct SubdMesh {
    std::vector<float3> P;                 // welded vertices
    std::vector<int> fv;                   // 3 per face
    std::vector<float2> fuv;               // 3 per face (corner uvs)
    std::vector<int> adj;                  // 3 per face: neighbour across edge k (v[k] -> v[k+1]) or -1
};

inline int nxt(int k) { return (k + 1) % 3; }
inline int prv(int k) { return (k + 2) % 3; }

void link_faces(SubdMesh& m) {
    const int nf = (int)m.fv.size() / 3;
    m.adj.assign(3 * (size_t)nf, -1);
    std::map<std::pair<int, int>, int> open;   // edge -> face * 3 + edge number
    for (int f = 0; f < nf; ++f)
        for (int k = 0; k < 3; ++k) {
            const int a = m.fv[3 * f + k], b = m.fv[3 * f + nxt(k)];
            const auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = open.find(key);
            if (it == open.end()) {
                open.emplace(key, 3 * f + k);
            } else {
                const int g = it->second / 3, e = it->second % 3;
                m.adj[3 * (size_t)g + e] = f;
                m.adj[3 * (size_t)f + k] = g;
                open.erase(it);           // a third face on this edge starts a new pair (boundary)
            }
        }
}

int corner_of(const SubdMesh& m, int f, int v) {
    for (int k = 0; k < 3; ++k) if (m.fv[3 * f + k] == v) return k;
    return -1;
}

// One-ring of every vertex in the order LoopSubdivMesh walks it (SDVertex::oneRing):
// interior vertices around their faces, boundary vertices from one boundary
// neighbour to the other. ring_face[i][j]: a face holding vertex i and ring vertex j.
struct Rings {
    std::vector<std::vector<int>> ring, faces;
    std::vector<char> boundary, used;
};

Rings build_rings(const SubdMesh& m) {
    const int nv = (int)m.P.size(), nf = (int)m.fv.size() / 3;
    Rings r;
    r.ring.assign(nv, {});
    r.faces.assign(nv, {});
    r.boundary.assign(nv, 0);
    r.used.assign(nv, 0);
    std::vector<int> start(nv, -1);
    for (int f = 0; f < nf; ++f)
        for (int k = 0; k < 3; ++k) { start[m.fv[3 * f + k]] = f; r.used[m.fv[3 * f + k]] = 1; }
    for (int v = 0; v < nv; ++v) {
        if (start[v] < 0) continue;
        // walk "next face" (across edge v -> nextVert) until it returns or runs out
        int f = start[v];
        int guard = 0;
        while (true) {
            const int k = corner_of(m, f, v);
            const int g = m.adj[3 * f + k];
            if (g < 0) { r.boundary[v] = 1; break; }
            f = g;
            if (f == start[v] || ++guard > nf) break;
        }
        if (!r.boundary[v]) {
            f = start[v];
            guard = 0;
            do {
                const int k = corner_of(m, f, v);
                r.ring[v].push_back(m.fv[3 * f + nxt(k)]);
                r.faces[v].push_back(f);
                f = m.adj[3 * f + k];
            } while (f >= 0 && f != start[v] && ++guard <= nf);
        } else {
            // f is the last face in the "next" direction; ring: its nextVert, then prevVerts
            const int k0 = corner_of(m, f, v);
            r.ring[v].push_back(m.fv[3 * f + nxt(k0)]);
            r.faces[v].push_back(f);
            guard = 0;
            while (f >= 0 && ++guard <= nf + 1) {
                const int k = corner_of(m, f, v);
                r.ring[v].push_back(m.fv[3 * f + prv(k)]);
                r.faces[v].push_back(f);
                f = m.adj[3 * f + prv(k)];
            }
        }
    }
    return r;
}

float beta_of(int n) { return n == 3 ? 3.f / 16.f : 3.f / (8.f * (float)n); }

SubdMesh weld(const Corners& cs) {
    SubdMesh m;
    std::map<std::tuple<float, float, float>, int> ids;
    const size_t nc = cs.P.size();
    for (size_t t = 0; t + 2 < nc; t += 3) {
        int id[3];
        for (int k = 0; k < 3; ++k) {
            const float3 p = cs.P[t + k];
            auto key = std::make_tuple(p.x, p.y, p.z);
            auto it = ids.find(key);
            if (it == ids.end()) { it = ids.emplace(key, (int)m.P.size()).first; m.P.push_back(p); }
            id[k] = it->second;
        }
        if (id[0] == id[1] || id[0] == id[2] || id[1] == id[2]) continue;   // degenerate: skipped
        for (int k = 0; k < 3; ++k) {
            m.fv.push_back(id[k]);
            m.fuv.push_back(cs.has_uv ? cs.UV[t + k] : make_float2(0.f, 0.f));
        }
    }
    link_faces(m);
    return m;
}

bool uv_eq(float2 a, float2 b) { return a.x == b.x && a.y == b.y; }

SubdMesh refine(const SubdMesh& m) {
    const int nv = (int)m.P.size(), nf = (int)m.fv.size() / 3;
    const Rings r = build_rings(m);
    SubdMesh out;
    out.P.resize(nv);
    // even vertices
    for (int v = 0; v < nv; ++v) {
        if (!r.used[v]) { out.P[v] = m.P[v]; continue; }
        const std::vector<int>& ring = r.ring[v];
        const int n = (int)ring.size();
        if (!r.boundary[v]) {
            const float b = beta_of(n);
            float3 p = scl(1.f - (float)n * b, m.P[v]);
            for (int j = 0; j < n; ++j) p = add(p, scl(b, m.P[ring[j]]));
            out.P[v] = p;
        } else {
            const float b = 1.f / 8.f;
            float3 p = scl(1.f - 2.f * b, m.P[v]);
            p = add(p, scl(b, m.P[ring[0]]));
            p = add(p, scl(b, m.P[ring[n - 1]]));
            out.P[v] = p;
        }
    }
    // per-vertex uv smoothness: all corners at the vertex agree, and every ring
    // neighbour has the same uv in the faces around it
    std::vector<char> uv_smooth(nv, 1);
    std::vector<float2> vuv(nv, make_float2(0.f, 0.f));
    std::vector<char> vuv_set(nv, 0);
    for (int f = 0; f < nf; ++f)
        for (int k = 0; k < 3; ++k) {
            const int v = m.fv[3 * f + k];
            if (!vuv_set[v]) { vuv[v] = m.fuv[3 * f + k]; vuv_set[v] = 1; }
            else if (!uv_eq(vuv[v], m.fuv[3 * f + k])) uv_smooth[v] = 0;
        }
    std::vector<char> even_uv_smooth(nv, 1);
    for (int v = 0; v < nv; ++v) {
        if (!r.used[v]) continue;
        even_uv_smooth[v] = uv_smooth[v];
        for (int j = 0; j < (int)r.ring[v].size() && even_uv_smooth[v]; ++j)
            if (!uv_smooth[r.ring[v][j]]) even_uv_smooth[v] = 0;
    }
    std::vector<float2> even_uv(nv, make_float2(0.f, 0.f));
    for (int v = 0; v < nv; ++v) {
        if (!r.used[v] || !even_uv_smooth[v]) continue;
        const std::vector<int>& ring = r.ring[v];
        const int n = (int)ring.size();
        if (!r.boundary[v]) {
            const float b = beta_of(n);
            float u = (1.f - (float)n * b) * vuv[v].x, w = (1.f - (float)n * b) * vuv[v].y;
            for (int j = 0; j < n; ++j) { u += b * vuv[ring[j]].x; w += b * vuv[ring[j]].y; }
            even_uv[v] = make_float2(u, w);
        } else {
            const float b = 1.f / 8.f;
            float u = (1.f - 2.f * b) * vuv[v].x, w = (1.f - 2.f * b) * vuv[v].y;
            u += b * (vuv[ring[0]].x + vuv[ring[n - 1]].x);
            w += b * (vuv[ring[0]].y + vuv[ring[n - 1]].y);
            even_uv[v] = make_float2(u, w);
        }
    }
    // odd vertices, one per edge (shared by the two faces)
    std::vector<int> odd(3 * (size_t)nf, -1);
    std::vector<float2> odd_uv(3 * (size_t)nf);
    for (int f = 0; f < nf; ++f)
        for (int k = 0; k < 3; ++k) {
            if (odd[3 * f + k] >= 0) continue;
            const int v0 = m.fv[3 * f + k], v1 = m.fv[3 * f + nxt(k)];
            const int g = m.adj[3 * f + k];
            const float2 u0 = m.fuv[3 * f + k], u1 = m.fuv[3 * f + nxt(k)];
            float3 p;
            const int id = (int)out.P.size();
            int ge = -1;
            if (g < 0) {
                p = scl(0.5f, add(m.P[v0], m.P[v1]));
                odd_uv[3 * f + k] = make_float2(0.5f * (u0.x + u1.x), 0.5f * (u0.y + u1.y));
            } else {
                ge = -1;
                for (int e = 0; e < 3; ++e) if (m.adj[3 * g + e] == f) { ge = e; break; }
                const int ov1 = m.fv[3 * f + prv(k)];
                const int gk0 = corner_of(m, g, v0), gk1 = corner_of(m, g, v1);
                int ov2 = m.fv[3 * g + 0];
                for (int e = 0; e < 3; ++e)
                    if (m.fv[3 * g + e] != v0 && m.fv[3 * g + e] != v1) ov2 = m.fv[3 * g + e];
                p = scl(3.f / 8.f, add(m.P[v0], m.P[v1]));
                p = add(p, scl(1.f / 8.f, add(m.P[ov1], m.P[ov2])));
                const bool uv_same = gk0 >= 0 && gk1 >= 0 && uv_eq(m.fuv[3 * g + gk0], u0) && uv_eq(m.fuv[3 * g + gk1], u1);
                if (uv_same) {
                    int go = 0;
                    for (int e = 0; e < 3; ++e) if (m.fv[3 * g + e] == ov2) go = e;
                    const float2 a = m.fuv[3 * f + prv(k)], b = m.fuv[3 * g + go];
                    const float2 s = make_float2(3.f / 8.f * (u0.x + u1.x) + 1.f / 8.f * (a.x + b.x),
                                                 3.f / 8.f * (u0.y + u1.y) + 1.f / 8.f * (a.y + b.y));
                    odd_uv[3 * f + k] = s;
                    if (ge >= 0) odd_uv[3 * g + ge] = s;
                } else {
                    odd_uv[3 * f + k] = make_float2(0.5f * (u0.x + u1.x), 0.5f * (u0.y + u1.y));
                    if (ge >= 0) {
                        const float2 a = m.fuv[3 * g + ge], b = m.fuv[3 * g + nxt(ge)];
                        odd_uv[3 * g + ge] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
                    }
                }
            }
            out.P.push_back(p);
            odd[3 * f + k] = id;
            if (ge >= 0) odd[3 * g + ge] = id;
        }
    // children in the reference's order: corner triangles 0, 1, 2, then the centre one
    out.fv.reserve(12 * (size_t)nf);
    out.fuv.reserve(12 * (size_t)nf);
    for (int f = 0; f < nf; ++f) {
        int ov[3];
        float2 ouv[3], cuv[3];
        for (int k = 0; k < 3; ++k) {
            ov[k] = odd[3 * f + k];
            ouv[k] = odd_uv[3 * f + k];
            const int v = m.fv[3 * f + k];
            cuv[k] = even_uv_smooth[v] ? even_uv[v] : m.fuv[3 * f + k];
        }
        for (int k = 0; k < 3; ++k) {
            int c[3];
            float2 cu[3];
            c[k] = m.fv[3 * f + k];      cu[k] = cuv[k];
            c[nxt(k)] = ov[k];           cu[nxt(k)] = ouv[k];
            c[prv(k)] = ov[prv(k)];      cu[prv(k)] = ouv[prv(k)];
            for (int e = 0; e < 3; ++e) { out.fv.push_back(c[e]); out.fuv.push_back(cu[e]); }
        }
        for (int k = 0; k < 3; ++k) { out.fv.push_back(ov[k]); out.fuv.push_back(ouv[k]); }
    }
    link_faces(out);
    return out;
}

// Limit positions and limit normals (loopSubdivMesh.cpp:434-530).
void to_limit(SubdMesh& m, std::vector<float3>* normals) {
    const int nv = (int)m.P.size();
    const Rings r = build_rings(m);
    std::vector<float3> lim(nv);
    for (int v = 0; v < nv; ++v) {
        if (!r.used[v]) { lim[v] = m.P[v]; continue; }
        const std::vector<int>& ring = r.ring[v];
        const int n = (int)ring.size();
        if (!r.boundary[v]) {
            const float g = 1.f / ((float)n + 3.f / (8.f * beta_of(n)));
            float3 p = scl(1.f - (float)n * g, m.P[v]);
            for (int j = 0; j < n; ++j) p = add(p, scl(g, m.P[ring[j]]));
            lim[v] = p;
        } else {
            const float b = 1.f / 5.f;
            float3 p = scl(1.f - 2.f * b, m.P[v]);
            p = add(p, scl(b, m.P[ring[0]]));
            p = add(p, scl(b, m.P[ring[n - 1]]));
            lim[v] = p;
        }
    }
    m.P = lim;
    normals->assign(nv, f3(0, 1, 0));
    for (int v = 0; v < nv; ++v) {
        if (!r.used[v]) continue;
        const std::vector<int>& ring = r.ring[v];
        const int n = (int)ring.size();
        float3 S = f3(0, 0, 0), T = f3(0, 0, 0);
        if (!r.boundary[v]) {
            for (int k = 0; k < n; ++k) {
                S = add(S, scl(cosf((float)(2.f * M_PI * k / n)), m.P[ring[k]]));
                T = add(T, scl(sinf((float)(2.f * M_PI * k / n)), m.P[ring[k]]));
            }
        } else {
            S = sub(m.P[ring[n - 1]], m.P[ring[0]]);
            if (n == 2) T = sub(add(m.P[ring[0]], m.P[ring[1]]), scl(2.f, m.P[v]));
            else if (n == 3) T = sub(m.P[ring[1]], m.P[v]);
            else if (n == 4)   // regular boundary vertex; summed left to right as the reference
                T = add(add(add(add(scl(-1.f, m.P[ring[0]]), scl(2.f, m.P[ring[1]])), scl(2.f, m.P[ring[2]])),
                            scl(-1.f, m.P[ring[3]])), scl(-2.f, m.P[v]));
            else {
                const float theta = (float)(M_PI / (float)(n - 1));
                T = scl(sinf(theta), add(m.P[ring[0]], m.P[ring[n - 1]]));
                for (int k = 1; k < n - 1; ++k) {
                    const float wt = (2.f * cosf(theta) - 2.f) * sinf((float)k * theta);
                    T = add(T, scl(wt, m.P[ring[k]]));
                }
                T = scl(-1.f, T);
            }
        }
        (*normals)[v] = nrm(crs(T, S));
    }
}

// ------------------------------------------------------------------ textures (PFM)
void read_pfm(const std::string& path, std::vector<float>* rgb, int* w, int* h) {
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) throw_load(AUR_ERR_IO, "cannot open texture " + path);
    char magic[3] = {0, 0, 0};
    double scale = 0.0;
    int ww = 0, hh = 0;
    const bool ok = fscanf(fp, "%2s %d %d %lf", magic, &ww, &hh, &scale) == 4 && fgetc(fp) != EOF;
    const int ch = ok && strcmp(magic, "PF") == 0 ? 3 : ok && strcmp(magic, "Pf") == 0 ? 1 : 0;
    if (!ch || ww <= 0 || hh <= 0 || (long long)ww * hh > (1ll << 28)) {
        fclose(fp);
        throw_load(AUR_ERR_PARSE, "not a PFM texture: " + path);
    }
    std::vector<float> data((size_t)ww * hh * ch);
    const size_t got = fread(data.data(), sizeof(float), data.size(), fp);
    fclose(fp);
    if (got != data.size()) throw_load(AUR_ERR_PARSE, "truncated PFM texture: " + path);
    if (scale > 0.0)   // big-endian samples
        for (float& f : data) {
            uint32_t u;
            memcpy(&u, &f, 4);
            u = (u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24);
            memcpy(&f, &u, 4);
        }
    // PFM rows run bottom to top; textures are stored top row first (Texture2D reads row
    // floor((1 - v) * height))
    rgb->resize((size_t)ww * hh * 3);
    for (int y = 0; y < hh; ++y)
        for (int x = 0; x < ww; ++x)
            for (int c = 0; c < 3; ++c)
                (*rgb)[3 * ((size_t)y * ww + x) + c] = data[((size_t)(hh - 1 - y) * ww + x) * ch + (ch == 3 ? c : 0)];
    *w = ww;
    *h = hh;
}

// A texture image: OpenEXR (what the reference reads) or PFM, by extension.
void read_image(const std::string& path, std::vector<float>* rgb, int* w, int* h) {
    const size_t dot = path.find_last_of('.');
    std::string ext = dot == std::string::npos ? "" : path.substr(dot);
    for (char& c : ext) c = (char)tolower((unsigned char)c);
    if (ext == ".exr") {
        std::string err;
        const aur_status st = read_exr_rgb(path, rgb, w, h, &err);
        if (st != AUR_OK) throw_load(st, err);
        return;
    }
    if (ext != ".pfm") throw_load(AUR_ERR_UNSUPPORTED, "texture " + path + " is neither OpenEXR nor PFM");
    read_pfm(path, rgb, w, h);
}

// ------------------------------------------------------------------ loader
std::string dir_of(const std::string& p) {
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string(".") : p.substr(0, s);
}
std::string resolve(const std::string& dir, const std::string& p) {
    if (p.empty() || p[0] == '/') return p;
    return dir + "/" + p;
}

struct Loader {
    aur_scene_file& out;
    std::string dir;
    std::map<std::string, int> textures;     // shader name -> texture index
    std::map<std::string, int> materials;    // material name -> index

    int texture_of(const std::string& shader, const std::string& where) {
        auto it = textures.find(shader);
        if (it == textures.end()) throw_load(AUR_ERR_PARSE, where + ": unknown shader \"" + shader + "\"");
        return it->second;
    }
    // A colour attribute: a constant [r, g, b] or the name of a colour shader
    void color_attr(const JValue& o, const char* key, float* rgb, int32_t* tex, const std::string& where) {
        const JValue& v = need(o, key, where);
        if (v.kind == JValue::Str) {
            if (!tex) throw_load(AUR_ERR_UNSUPPORTED, where + ": \"" + key + "\" cannot be a shader in this build");
            *tex = texture_of(v.str, where);
            return;
        }
        double c[3];
        need_nums(o, key, 3, c, where);
        for (int i = 0; i < 3; ++i) rgb[i] = (float)c[i];
    }
    void float_attr(const JValue& o, const char* key, float* val, int32_t* tex, const std::string& where) {
        const JValue& v = need(o, key, where);
        if (v.kind == JValue::Str) {
            if (!tex) throw_load(AUR_ERR_UNSUPPORTED, where + ": \"" + key + "\" cannot be a shader in this build");
            *tex = texture_of(v.str, where);
            return;
        }
        *val = (float)need_num(o, key, where);
    }

    void shaders(const JValue& root) {
        const JValue* s = root.get("shaders");
        if (!s) return;
        if (s->kind != JValue::Obj) throw_load(AUR_ERR_PARSE, "\"shaders\" must be an object");
        for (const auto& kv : s->obj) {
            const std::string where = "shader \"" + kv.first + "\"";
            const std::string at = need_str(kv.second, "attributetype", where);
            if (at != "color" && at != "float") throw_load(AUR_ERR_PARSE, where + ": unknown attributetype " + at);
            const std::string type = need_str(kv.second, "type", where);
            float scale = 0.f;
            if (type == "triplanarTextureShader") {           // jsonParser.cpp:547-551, 568-572
                scale = (float)need_num(kv.second, "scale", where);
                if (!(scale > 0.f) || !std::isfinite(scale))
                    throw_load(AUR_ERR_PARSE, where + ": triplanar scale must be a finite number > 0");
            } else if (type != "texture2DShader") {
                throw_load(AUR_ERR_PARSE, where + ": unknown shader type " + type);
            }
            const std::string path = resolve(dir, need_str(kv.second, "texturename", where));
            std::vector<float> rgb;
            int w = 0, h = 0;
            read_image(path, &rgb, &w, &h);
            textures[kv.first] = (int)out.tex_dims.size() / 2;
            out.tex_dims.push_back(w);
            out.tex_dims.push_back(h);
            out.tex_scale.push_back(scale);
            out.texels.insert(out.texels.end(), rgb.begin(), rgb.end());
        }
    }

    // getMaterial (jsonParser.cpp:313-429)
    void materials_(const JValue& root) {
        const JValue* s = root.get("materials");
        if (!s) return;
        if (s->kind != JValue::Obj) throw_load(AUR_ERR_PARSE, "\"materials\" must be an object");
        for (const auto& kv : s->obj) {
            const std::string where = "material \"" + kv.first + "\"";
            const JValue& o = kv.second;
            const std::string type = need_str(o, "type", where);
            aur_material_desc m;
            memset(&m, 0, sizeof(m));
            m.diffuse_tex = m.specular_tex = m.roughness_tex = -1;
            m.normal_kind = AUR_NORMAL_NONE;
            m.normal_tex = -1;
            if (o.get("normalmap")) {                        // getMaterial (jsonParser.cpp:317-322)
                color_attr(o, "normalmap", m.normal, &m.normal_tex, where);
                m.normal_kind = m.normal_tex >= 0 ? AUR_NORMAL_TEXTURE : AUR_NORMAL_CONSTANT;
            }
            m.gain[0] = m.gain[1] = m.gain[2] = 1.f;
            m.ior = 1.f;
            if (type == "matteMaterial") {
                m.type = AUR_MAT_MATTE;
                color_attr(o, "color", m.diffuse, &m.diffuse_tex, where);
            } else if (type == "kelemenMaterial") {
                m.type = AUR_MAT_KELEMEN;
                color_attr(o, "diffusecolor", m.diffuse, &m.diffuse_tex, where);
                color_attr(o, "speccolor", m.specular, &m.specular_tex, where);
                float_attr(o, "reflectance", &m.reflectance, nullptr, where);   // a constant in the reference too
                float_attr(o, "roughness", &m.roughness, &m.roughness_tex, where);
            } else if (type == "metalMaterial") {
                m.type = AUR_MAT_METAL;
                color_attr(o, "reflectance", m.specular, nullptr, where);
                float_attr(o, "roughnessA", &m.roughness, nullptr, where);
                float_attr(o, "roughnessB", &m.roughness_b, nullptr, where);
                float_attr(o, "mix", &m.mix, nullptr, where);
                color_attr(o, "gain", m.gain, nullptr, where);
            } else if (type == "glassMaterial") {   // constants only, as the reference reads them
                m.type = AUR_MAT_GLASS;
                color_attr(o, "specColor", m.specular, nullptr, where);
                color_attr(o, "transmitColor", m.diffuse, nullptr, where);
                float_attr(o, "reflectance", &m.reflectance, nullptr, where);
                float_attr(o, "ior", &m.ior, nullptr, where);
            } else if (type == "carMaterial") {   // its construction is commented out in jsonParser.cpp:369-415
                throw_load(AUR_ERR_UNSUPPORTED, where + ": carMaterial is disabled in the reference's parser");
            } else {
                throw_load(AUR_ERR_PARSE, where + ": unknown material type " + type);
            }
            materials[kv.first] = (int)out.materials.size();
            out.materials.push_back(m);
        }
    }

    // AttributeState::cameraToObject of an attribute: the inverse its Transform carries
    void push_c2o(const Xform& o2c) {
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) out.attr_c2o.push_back(o2c.inv.m[i][j]);
    }

    void append_mesh(const std::vector<float3>& P, const std::vector<int>& idx, const std::vector<float3>& Ncorner,
                     const std::vector<float2>& UVcorner, int attr) {
        const uint32_t base = (uint32_t)(out.verts.size() / 3);
        for (const float3& p : P) { out.verts.push_back(p.x); out.verts.push_back(p.y); out.verts.push_back(p.z); }
        const size_t nt = idx.size() / 3;
        for (size_t t = 0; t < nt; ++t) {
            for (int k = 0; k < 3; ++k) {
                out.tri_vidx.push_back(base + (uint32_t)idx[3 * t + k]);
                const float3 n = Ncorner[3 * t + k];
                out.corner_normals.push_back(n.x); out.corner_normals.push_back(n.y); out.corner_normals.push_back(n.z);
                const float2 u = UVcorner.empty() ? make_float2(0.f, 0.f) : UVcorner[3 * t + k];
                out.corner_uvs.push_back(u.x); out.corner_uvs.push_back(u.y);
            }
            out.tri_attr.push_back(attr);
        }
    }

    // getGeometry + ObjTriangleMesh + TriangleMesh::makeEmbree (triangleMesh.cpp:57-81)
    void geometry(const JValue& o, const std::string& key, const Xform& inv_cam, int attr) {
        const std::string where = "object \"" + key + "\"";
        const std::string path = resolve(dir, need_str(o, "path", where));
        const std::string mat = need_str(o, "material", where);
        const Xform o2c = inv_cam * parse_transforms(o.get("transforms"), where);
        const int levels = (int)need_num(o, "subdlevels", where);
        if (levels < 0 || levels > 8) throw_load(AUR_ERR_PARSE, where + ": subdlevels must be 0..8");
        auto mit = materials.find(mat);
        if (mit == materials.end()) throw_load(AUR_ERR_PARSE, where + ": unknown material \"" + mat + "\"");
        out.attr_material.push_back(mit->second);
        out.attr_emission.insert(out.attr_emission.end(), {0.f, 0.f, 0.f});
        push_c2o(o2c);
        const Corners cs = read_obj(path);
        std::vector<float3> P, N;
        std::vector<float2> UV;
        std::vector<int> idx;
        if (levels == 0) {
            // per-corner vertices, as ObjTriangleMesh hands them to TriangleMesh
            for (size_t i = 0; i < cs.P.size(); ++i) {
                P.push_back(o2c.point(cs.P[i]));
                N.push_back(o2c.vector(cs.N[i]));
                idx.push_back((int)i);
                if (cs.has_uv) UV.push_back(cs.UV[i]);
            }
        } else {
            SubdMesh m = weld(cs);
            for (int l = 0; l < levels; ++l) m = refine(m);
            std::vector<float3> vn;
            to_limit(m, &vn);
            for (const float3& p : m.P) P.push_back(o2c.point(p));
            for (size_t c = 0; c < m.fv.size(); ++c) {
                idx.push_back(m.fv[c]);
                N.push_back(o2c.vector(vn[m.fv[c]]));
                if (cs.has_uv) UV.push_back(m.fuv[c]);
            }
        }
        append_mesh(P, idx, N, UV, attr);
    }

    // getLight + SquareLight (jsonParser.cpp:240-260, squareLight.cpp:20-52, :78-94)
    void light(const JValue& o, const std::string& key, const Xform& inv_cam, int attr) {
        const std::string where = "light \"" + key + "\"";
        const Xform o2c = inv_cam * parse_transforms(o.get("transforms"), where);
        aur_light_desc l;
        memset(&l, 0, sizeof(l));
        l.type = AUR_LIGHT_SQUARE;
        l.tex = -1;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) l.object_to_camera[4 * i + j] = o2c.m.m[i][j];
        l.size_x = (float)need_num(o, "scaleX", where);
        l.size_y = (float)need_num(o, "scaleY", where);
        l.exposure = (float)need_num(o, "exposure", where);
        double c[3];
        need_nums(o, "color", 3, c, where);
        for (int i = 0; i < 3; ++i) l.color[i] = (float)c[i];
        out.lights.push_back(l);
        const float sx = l.size_x, sy = l.size_y;
        const float3 p[4] = {o2c.point(f3(-sx, -sy, 0)), o2c.point(f3(-sx, sy, 0)), o2c.point(f3(sx, sy, 0)),
                             o2c.point(f3(sx, -sy, 0))};
        const float3 ln = nrm(crs(sub(p[0], p[1]), sub(p[1], p[2])));
        const float3 n = o2c.vector(ln);    // makeEmbree transforms the shape's normal again
        const std::vector<float3> P(p, p + 4);
        const std::vector<int> idx = {0, 1, 3, 2, 1, 3};
        const std::vector<float3> N(6, n);
        append_mesh(P, idx, N, {}, attr);
        const float inten = powf(2.f, l.exposure);
        out.attr_emission.insert(out.attr_emission.end(), {l.color[0] * inten, l.color[1] * inten, l.color[2] * inten});
        push_c2o(o2c);
    }

    // getEnvLight + InfiniteAreaLight (jsonParser.cpp:262-280, infiniteAreaLight.cpp:21-33): the
    // map is looked up in world directions through the camera-to-world transform
    void env_light(const JValue& o, const std::string& key, const Xform& cam_to_world, int attr) {
        const std::string where = "envlight \"" + key + "\"";
        parse_transforms(o.get("transforms"), where);   // read and checked, as the reference reads them
        aur_light_desc l;
        memset(&l, 0, sizeof(l));
        l.type = AUR_LIGHT_ENV;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) l.object_to_camera[4 * i + j] = cam_to_world.m.m[i][j];
        l.exposure = (float)need_num(o, "exposure", where);
        double c[3];
        need_nums(o, "color", 3, c, where);
        for (int i = 0; i < 3; ++i) l.color[i] = (float)c[i];
        l.tex = -1;
        const std::string map = need_str(o, "envmap", where);
        if (!map.empty()) {
            const std::string path = resolve(dir, map);
            std::vector<float> rgb;
            int w = 0, h = 0;
            read_image(path, &rgb, &w, &h);
            l.tex = (int32_t)(out.tex_dims.size() / 2);
            out.tex_dims.push_back(w);
            out.tex_dims.push_back(h);
            out.tex_scale.push_back(0.f);
            out.texels.insert(out.texels.end(), rgb.begin(), rgb.end());
        }
        out.lights.push_back(l);
        out.attr_emission.insert(out.attr_emission.end(), {1.f, 1.f, 1.f});   // InfiniteAreaLight::emission()
        push_c2o(Xform());
        (void)attr;
    }

    void load(const std::string& path) {
        std::ifstream in(path, std::ios::binary);
        if (!in) throw_load(AUR_ERR_IO, "cannot open scene file " + path);
        std::stringstream ss;
        ss << in.rdbuf();
        const std::string text = ss.str();
        JParser jp;
        jp.begin = jp.p = text.data();
        jp.end = text.data() + text.size();
        JValue root;
        if (!jp.value(root, 0)) throw_load(AUR_ERR_PARSE, path + ": " + jp.err);
        jp.ws();
        if (jp.p != jp.end) { jp.fail("trailing characters"); throw_load(AUR_ERR_PARSE, path + ": " + jp.err); }
        if (root.kind != JValue::Obj || root.obj.empty()) throw_load(AUR_ERR_PARSE, path + ": no keys in the scene file");
        dir = dir_of(path);
        // options (parseOptions, jsonParser.cpp:432-474)
        const JValue* opt = root.get("options");
        if (!opt) throw_load(AUR_ERR_PARSE, "no \"options\"");
        double res[2];
        need_nums(*opt, "resolution", 2, res, "options");
        out.width = (int32_t)res[0];
        out.height = (int32_t)res[1];
        if (out.width <= 0 || out.height <= 0) throw_load(AUR_ERR_PARSE, "options: bad resolution");
        memset(&out.opts, 0, sizeof(out.opts));
        out.opts.spp = (int32_t)need_num(*opt, "pixelsamples", "options");
        out.light_samples = (int32_t)need_num(*opt, "lightsamples", "options");
        out.opts.min_depth = (int32_t)need_num(*opt, "mindepth", "options");
        out.opts.max_depth = (int32_t)need_num(*opt, "maxdepth", "options");
        out.opts.mode = AUR_RENDER_WAVEFRONT;
        out.opts.wf_sort = -1;
        if (out.light_samples < 1) throw_load(AUR_ERR_PARSE, "options: lightsamples must be >= 1");
        out.opts.light_samples = out.light_samples;
        out.output = need_str(*opt, "filename", "options");
        // camera (parseCamera, jsonParser.cpp:476-502)
        const JValue* cam = root.get("renderCam");
        if (!cam) throw_load(AUR_ERR_PARSE, "no \"renderCam\"");
        out.fov = (float)need_num(*cam, "fov", "renderCam");
        const Xform cam_to_world = parse_transforms(cam->get("transforms"), "renderCam");
        const Xform inv_cam = cam_to_world.inverted();
        shaders(root);
        materials_(root);
        // objects (parseGeometry, jsonParser.cpp:602-648): geometry first, then light shapes
        const JValue* objs = root.get("objects");
        if (!objs || objs->kind != JValue::Obj) throw_load(AUR_ERR_PARSE, "no \"objects\"");
        std::vector<std::pair<std::string, const JValue*>> geo, lights;
        for (const auto& kv : objs->obj) {
            const std::string type = need_str(kv.second, "type", "object \"" + kv.first + "\"");
            if (type == "geometry") geo.emplace_back(kv.first, &kv.second);
            else if (type == "light") lights.emplace_back(kv.first, &kv.second);
            else if (type == "envlight") lights.emplace_back(kv.first, &kv.second);
            // unknown types are skipped, as the reference warns and skips them
        }
        if (geo.empty()) throw_load(AUR_ERR_PARSE, "no geometry objects");
        int attr = 0;
        for (auto& g : geo) geometry(*g.second, g.first, inv_cam, attr++);
        const int constant = (int)out.materials.size();
        aur_material_desc black;
        memset(&black, 0, sizeof(black));
        black.type = AUR_MAT_CONSTANT;
        black.diffuse_tex = black.specular_tex = black.roughness_tex = black.normal_tex = -1;
        black.gain[0] = black.gain[1] = black.gain[2] = 1.f;
        black.ior = 1.f;
        out.materials.push_back(black);
        for (auto& l : lights) {
            out.attr_material.push_back(constant);
            if (need_str(*l.second, "type", "object") == "envlight") env_light(*l.second, l.first, cam_to_world, attr++);
            else light(*l.second, l.first, inv_cam, attr++);
        }
        if (out.tri_vidx.size() / 3 >= (1u << 30)) throw_load(AUR_ERR_UNSUPPORTED, "more than 2^30 triangles");
    }
};

}  // namespace
}  // namespace aur

using namespace aur;

extern "C" {

aur_status aur_scene_file_read(const char* path, aur_scene_file** out) {
    if (!path || !out) return fail(AUR_ERR_INVALID_ARG, "aur_scene_file_read: NULL argument");
    *out = nullptr;
    aur_scene_file* f = new (std::nothrow) aur_scene_file();
    if (!f) return fail(AUR_ERR_OOM, "aur_scene_file_read: out of host memory");
    try {
        Loader ld{*f, "", {}, {}};
        ld.load(path);
    } catch (const LoadError& e) {
        delete f;
        return fail(e.status, std::string("aur_scene_file_read: ") + e.msg);
    } catch (const std::bad_alloc&) {
        delete f;
        return fail(AUR_ERR_OOM, "aur_scene_file_read: out of host memory");
    }
    *out = f;
    return AUR_OK;
}

aur_status aur_scene_file_desc(const aur_scene_file* f, aur_scene_desc* d, aur_render_opts* opts) {
    if (!f || !d) return fail(AUR_ERR_INVALID_ARG, "aur_scene_file_desc: NULL argument");
    memset(d, 0, sizeof(*d));
    d->verts = f->verts.data();
    d->nvert = (uint32_t)(f->verts.size() / 3);
    d->tri_vidx = f->tri_vidx.data();
    d->tri_attr = f->tri_attr.data();
    d->corner_normals = f->corner_normals.data();
    d->corner_uvs = f->corner_uvs.data();
    d->ntri = (uint32_t)f->tri_attr.size();
    d->attr_material = f->attr_material.data();
    d->attr_emission = f->attr_emission.data();
    d->nattr = (uint32_t)f->attr_material.size();
    d->materials = f->materials.data();
    d->nmat = (uint32_t)f->materials.size();
    d->lights = f->lights.empty() ? nullptr : f->lights.data();
    d->nlight = (uint32_t)f->lights.size();
    d->texels = f->texels.empty() ? nullptr : f->texels.data();
    d->tex_dims = f->tex_dims.empty() ? nullptr : f->tex_dims.data();
    d->ntex = (uint32_t)(f->tex_dims.size() / 2);
    d->tex_triplanar_scale = f->tex_scale.empty() ? nullptr : f->tex_scale.data();
    d->attr_camera_to_object = f->attr_c2o.empty() ? nullptr : f->attr_c2o.data();
    d->fov = f->fov;
    d->width = f->width;
    d->height = f->height;
    if (opts) *opts = f->opts;
    return AUR_OK;
}

const char* aur_scene_file_output(const aur_scene_file* f) { return f ? f->output.c_str() : ""; }

int32_t aur_scene_file_light_samples(const aur_scene_file* f) { return f ? f->light_samples : 0; }

aur_status aur_scene_file_destroy(aur_scene_file* f) {
    delete f;
    return AUR_OK;
}

aur_status aur_scene_load_json(aur_ctx* ctx, const char* path, const aur_bvh_opts* bvh_opts, aur_scene** out,
                               aur_render_opts* opts) {
    if (!ctx || !path || !out) return fail(AUR_ERR_INVALID_ARG, "aur_scene_load_json: NULL argument");
    *out = nullptr;
    aur_scene_file* f = nullptr;
    aur_status st = aur_scene_file_read(path, &f);
    if (st != AUR_OK) return st;
    aur_scene_desc d;
    aur_scene_file_desc(f, &d, opts);
    st = aur_scene_create(ctx, &d, bvh_opts, out);
    aur_scene_file_destroy(f);
    return st;
}

}  // extern "C"
