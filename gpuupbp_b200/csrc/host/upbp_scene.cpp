// OBJ + MTL + AUX scene loader with the reference's semantics
// (gpuupbp/misc/scene_loader_obj.cpp): MTL Kd/Ks/Ns/Ke; AUX camera (TM_ROW0-3,
// CAMERA_FOV in radians, CAMERA_MATERIAL), materials (geometryType, priority,
// mediumId, mirror, ior, Ke, enclosingMatId), media (absorption, scattering,
// emission, g, continuation_probability), globalMediumId and the extra lights
// (light_point, light_directional, light_background_constant,
// light_background_em with its OpenEXR environment map).  One area
// light per emissive triangle; lights listed in the AUX file come first.
// Also the camera matrices of gpuupbp/host/camera.hpp:33-76.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "upbp_scene.h"

namespace upbp_host {

static std::mutex g_err_mu;
static std::string g_err;

void set_error(const std::string& msg)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
}

const char* get_error()
{
    static thread_local std::string copy;
    std::lock_guard<std::mutex> lk(g_err_mu);
    copy = g_err;
    return copy.c_str();
}

namespace {

struct V3 {
    double x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// float versions used where the reference computes in single precision
struct F3 {
    float x, y, z;
};
F3 fsub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
F3 fcross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float fdot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
F3 fnormalize(F3 a)
{
    const float inv = 1.f / std::sqrt(fdot(a, a));
    return {a.x * inv, a.y * inv, a.z * inv};
}
F3 fneg(F3 a) { return {-a.x, -a.y, -a.z}; }

struct ObjMat {
    std::string name;
    float kd[3] = {0, 0, 0}, ks[3] = {0, 0, 0}, ke[3] = {0, 0, 0}, mirror[3] = {0, 0, 0};
    float ns = 0.f;
    bool emissive = false;
    int medium = -1, enclosing = -1, priority = -1;
    bool real = true;
    float ior = -1.f;
};

struct ObjMed {
    std::string name;
    float absorption[3] = {0, 0, 0}, emission[3] = {0, 0, 0}, scattering[3] = {.5f, .5f, .5f};
    float cont = -1.f, g = 0.f;
};

struct Tri {
    int v[3];
    int n[3];
    int mat;
};

struct AuxLight {
    int type;  // UPBP_LIGHT_*
    float pos[3] = {0, 0, 0}, emission[3] = {0, 0, 0};
    std::string env_map;  // light_background_em: image file
    float env_scale = 1.f, env_rotate = 0.f;
};

std::string dir_of(const std::string& p)
{
    const size_t i = p.find_last_of('/');
    return i == std::string::npos ? std::string() : p.substr(0, i + 1);
}

int find_mat(const std::vector<ObjMat>& m, const std::string& name)
{
    for (size_t i = 0; i < m.size(); i++)
        if (m[i].name == name) return (int)i;
    return -1;
}

int find_or_add_med(std::vector<ObjMed>& m, const std::string& name)
{
    for (size_t i = 0; i < m.size(); i++)
        if (m[i].name == name) return (int)i;
    ObjMed x;
    x.name = name;
    m.push_back(x);
    return (int)m.size() - 1;
}

bool read3(std::istringstream& ss, float* v) { return bool(ss >> v[0] >> v[1] >> v[2]); }

bool read_mtl(const std::string& path, std::vector<ObjMat>& mats)
{
    std::ifstream f(path);
    if (!f) {
        set_error("could not open " + path);
        return false;
    }
    std::string line;
    ObjMat* cur = nullptr;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string key;
        if (!(ss >> key) || key[0] == '#') continue;
        if (key == "newmtl") {
            std::string name;
            ss >> name;
            mats.push_back(ObjMat{});
            cur = &mats.back();
            cur->name = name;
        } else if (!cur) {
            continue;
        } else if (key == "Ns") {
            ss >> cur->ns;
        } else if (key == "Kd") {
            read3(ss, cur->kd);
        } else if (key == "Ks") {
            read3(ss, cur->ks);
        } else if (key == "Ke") {
            read3(ss, cur->ke);
            cur->emissive = cur->ke[0] > 0.f || cur->ke[1] > 0.f || cur->ke[2] > 0.f;
        }
    }
    return true;
}

// One face-vertex token: v, v/t, v//n or v/t/n; returns the format id.
int parse_fv(const std::string& t, int& v, int& n)
{
    n = -1;
    const size_t s1 = t.find('/');
    if (s1 == std::string::npos) {
        v = std::atoi(t.c_str());
        return 0;
    }
    v = std::atoi(t.substr(0, s1).c_str());
    const size_t s2 = t.find('/', s1 + 1);
    if (s2 == std::string::npos) return 1;           // v/t
    if (s2 == s1 + 1) {                               // v//n
        n = std::atoi(t.substr(s2 + 1).c_str());
        return 2;
    }
    n = std::atoi(t.substr(s2 + 1).c_str());          // v/t/n
    return 3;
}

}  // namespace

static void mat_mul(const float* a, const float* b, float* o)
{
    float r[16];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            float s = 0.f;
            for (int k = 0; k < 4; k++) s += a[i * 4 + k] * b[k * 4 + j];
            r[i * 4 + j] = s;
        }
    std::memcpy(o, r, sizeof(r));
}

static void mat_inverse(const float* m, float* out)
{
    double a[4][8];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 8; j++) a[i][j] = j < 4 ? m[i * 4 + j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++)
            if (std::fabs(a[r][c]) > std::fabs(a[p][c])) p = r;
        for (int j = 0; j < 8; j++) std::swap(a[c][j], a[p][j]);
        const double d = a[c][c];
        for (int j = 0; j < 8; j++) a[c][j] /= d;
        for (int r = 0; r < 4; r++) {
            if (r == c) continue;
            const double f = a[r][c];
            for (int j = 0; j < 8; j++) a[r][j] -= f * a[c][j];
        }
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out[i * 4 + j] = (float)a[i][j + 4];
}

static void mat_identity(float* m)
{
    for (int i = 0; i < 16; i++) m[i] = (i % 5 == 0) ? 1.f : 0.f;
}

CameraMatrices camera_setup(const upbp_camera_desc& c, float res_x, float res_y)
{
    CameraMatrices cm{};
    const F3 origin{c.origin[0], c.origin[1], c.origin[2]};
    const F3 target{c.target[0], c.target[1], c.target[2]};
    const F3 roll{c.roll[0], c.roll[1], c.roll[2]};
    const F3 fwd = fnormalize(fsub(target, origin));
    const F3 up = fnormalize(fcross(roll, fneg(fwd)));
    const F3 left = fcross(fneg(fwd), up);
    const F3 pos{fdot(up, origin), fdot(left, origin), fdot(fneg(fwd), origin)};
    float w2c[16];
    mat_identity(w2c);
    const F3 rows[3] = {up, left, fneg(fwd)};
    const float trans[3] = {-pos.x, -pos.y, -pos.z};
    for (int r = 0; r < 3; r++) {
        w2c[r * 4 + 0] = rows[r].x;
        w2c[r * 4 + 1] = rows[r].y;
        w2c[r * 4 + 2] = rows[r].z;
        w2c[r * 4 + 3] = trans[r];
    }
    const float fov = c.horizontal_fov_deg;
    const float f = 1.f / std::tan(fov * 3.14159265358979323846f / 360.f);
    const float nearp = 0.1f, farp = 10000.f;
    const float d = 1.f / (nearp - farp);
    float persp[16] = {f, 0, 0, 0, 0, -f, 0, 0, 0, 0, (nearp + farp) * d, 2.f * nearp * farp * d, 0, 0, -1.f, 0};
    float w2ns[16], ns2w[16];
    mat_mul(persp, w2c, w2ns);
    mat_inverse(w2ns, ns2w);
    const float aspect = res_x / res_y;
    float sc[16], tr[16], tmp[16];
    mat_identity(sc);
    sc[0] = res_x * .5f;
    sc[5] = res_x * .5f;
    sc[10] = 0.f;
    mat_identity(tr);
    tr[3] = 1.f;
    tr[7] = 1.f / aspect;
    tr[11] = 0.f;
    mat_mul(sc, tr, tmp);
    mat_mul(tmp, w2ns, cm.world_to_raster);
    float tr2[16], sc2[16];
    mat_identity(tr2);
    tr2[3] = -1.f;
    tr2[7] = -1.f / aspect;
    tr2[11] = 0.f;
    mat_identity(sc2);
    sc2[0] = 2.f / res_x;
    sc2[5] = 2.f / res_x;
    sc2[10] = 0.f;
    mat_mul(ns2w, tr2, tmp);
    mat_mul(tmp, sc2, cm.raster_to_world);
    const float th = std::tan(fov * 3.14159265358979323846f / 360.f);
    cm.image_plane_dist = res_x / (2.f * th);
    cm.origin[0] = origin.x;
    cm.origin[1] = origin.y;
    cm.origin[2] = origin.z;
    cm.direction[0] = fwd.x;
    cm.direction[1] = fwd.y;
    cm.direction[2] = fwd.z;
    return cm;
}

}  // namespace upbp_host

namespace upbp_host {

// The environment map of a background light: the image as the reference's
// tinyexr_wrapper::load_image leaves it (tinyexr_wrapper.cpp:97-136): every
// pixel times `scale`, columns shifted right by (int)(rotate * width) with
// wrap-around.  Shifts outside [0, width] are refused (the reference would
// write outside its image).
int load_env_map(const std::string& path, float rotate, float scale, upbp_scene& sc)
{
    int w = 0, h = 0;
    std::vector<float> in;
    std::string err;
    if (!read_exr_rgb(path, w, h, in, err)) {
        set_error("environment map: " + err);
        return UPBP_ERR_IO;
    }
    const int rot = (int)(rotate * (float)w);
    if (rot < 0 || rot > w) {
        set_error("environment map rotation must lie in [0, 1]");
        return UPBP_ERR_SCENE;
    }
    sc.env_rgb.assign(in.size(), 0.f);
    for (int j = 0; j < h; j++)
        for (int i = 0; i < w; i++) {
            int x = i + rot;
            if (x >= w) x -= w;
            for (int k = 0; k < 3; k++)
                sc.env_rgb[3 * ((size_t)j * w + x) + k] = in[3 * ((size_t)j * w + i) + k] * scale;
        }
    sc.env_width = (uint32_t)w;
    sc.env_height = (uint32_t)h;
    return UPBP_OK;
}

}  // namespace upbp_host

void upbp_scene::finalize()
{
    desc.triangle_count = (uint32_t)tri_material.size();
    desc.verts = verts.data();
    desc.normals = normals.data();
    desc.tri_material = tri_material.data();
    desc.tri_light = tri_light.data();
    desc.material_count = (uint32_t)materials.size();
    desc.materials = materials.data();
    desc.medium_count = (uint32_t)media.size();
    desc.media = media.data();
    desc.light_count = (uint32_t)lights.size();
    desc.lights = lights.data();
    desc.env_width = env_width;
    desc.env_height = env_height;
    desc.env_rgb = env_rgb.empty() ? nullptr : env_rgb.data();
    desc.sphere_count = (uint32_t)sph_material.size();
    desc.spheres = spheres.data();
    desc.sph_material = sph_material.data();
}

using namespace upbp_host;

extern "C" int upbp_scene_load_obj(const char* obj_path, uint32_t res_x, uint32_t res_y, upbp_scene** out)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!obj_path || !out || res_x == 0 || res_y == 0) return UPBP_ERR_ARGS;
        const std::string path = obj_path;
        std::ifstream f(path);
        if (!f) {
            set_error("could not open " + path);
            return UPBP_ERR_IO;
        }
        std::vector<float> v, vn;
        std::vector<ObjMat> mats;
        std::vector<ObjMed> meds;
        std::vector<Tri> tris;
        std::vector<int> group_mat_order;  // material of each usemtl group in order
        int cur_mat = -1;
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ss(line);
            std::string key;
            if (!(ss >> key) || key[0] == '#') continue;
            if (key == "v") {
                float x[3];
                read3(ss, x);
                v.insert(v.end(), x, x + 3);
            } else if (key == "vn") {
                float x[3];
                read3(ss, x);
                vn.insert(vn.end(), x, x + 3);
            } else if (key == "mtllib") {
                std::string name;
                ss >> name;
                if (!read_mtl(dir_of(path) + name, mats)) return UPBP_ERR_IO;
            } else if (key == "usemtl") {
                std::string name;
                ss >> name;
                cur_mat = find_mat(mats, name);
                if (cur_mat < 0) {
                    set_error("material not found: " + name);
                    return UPBP_ERR_SCENE;
                }
            } else if (key == "f") {
                if (cur_mat < 0) {
                    set_error("face before usemtl");
                    return UPBP_ERR_SCENE;
                }
                std::vector<std::string> toks;
                std::string t;
                while (ss >> t) toks.push_back(t);
                if (toks.size() < 3) continue;
                int fv[3], fn[3];
                const int fmt = parse_fv(toks[0], fv[0], fn[0]);
                parse_fv(toks[1], fv[1], fn[1]);
                parse_fv(toks[2], fv[2], fn[2]);
                const bool has_n = fmt == 2 || fmt == 3;
                Tri tr;
                for (int k = 0; k < 3; k++) {
                    tr.v[k] = fv[k] - 1;
                    tr.n[k] = has_n ? fn[k] - 1 : -1;
                }
                tr.mat = cur_mat;
                tris.push_back(tr);
                for (size_t k = 3; k < toks.size(); k++) {
                    int nv, nn;
                    parse_fv(toks[k], nv, nn);
                    Tri t2;
                    t2.v[0] = tris.back().v[0];
                    t2.n[0] = tris.back().n[0];
                    t2.v[1] = tris.back().v[2];
                    t2.n[1] = tris.back().n[2];
                    t2.v[2] = nv - 1;
                    t2.n[2] = has_n ? nn - 1 : -1;
                    t2.mat = cur_mat;
                    tris.push_back(t2);
                }
            }
        }

        // AUX file
        std::ifstream fa(path + ".aux");
        if (!fa) {
            set_error("could not open " + path + ".aux");
            return UPBP_ERR_IO;
        }
        float tm[4][3] = {{0}};
        float fov_rad = 0.f, focal = 1.f;
        int cam_mat = -1;
        int global_med = -1;
        std::vector<AuxLight> aux_lights;
        ObjMat* mat = nullptr;
        int med = -1;
        while (std::getline(fa, line)) {
            std::istringstream ss(line);
            std::string key;
            if (!(ss >> key) || key[0] == '#') continue;
            if (key.compare(0, 6, "TM_ROW") == 0 && key.size() == 7) {
                const int r = key[6] - '0';
                if (r >= 0 && r < 4) read3(ss, tm[r]);
            } else if (key == "CAMERA_FOV") {
                ss >> fov_rad;
            } else if (key == "CAMERA_TDIST") {
                ss >> focal;
            } else if (key == "CAMERA_MATERIAL") {
                std::string name;
                ss >> name;
                cam_mat = find_mat(mats, name);
                if (cam_mat < 0) {
                    set_error("material not found: " + name);
                    return UPBP_ERR_SCENE;
                }
            } else if (key == "CAMERA_RESOLUTION_X" || key == "CAMERA_RESOLUTION_Y") {
                // the command line decides the resolution
            } else if (key == "material") {
                std::string name;
                ss >> name;
                const int m = find_mat(mats, name);
                if (m < 0) {
                    set_error("material not found: " + name);
                    return UPBP_ERR_SCENE;
                }
                mat = &mats[m];
            } else if (key == "medium") {
                std::string name;
                ss >> name;
                med = find_or_add_med(meds, name);
            } else if (key == "mediumId" || key == "mirror" || key == "ior" || key == "priority" ||
                       key == "geometryType" || key == "Ke" || key == "enclosingMatId") {
                if (!mat) {
                    set_error("using " + key + " option without material selection");
                    return UPBP_ERR_SCENE;
                }
                if (key == "mediumId") {
                    std::string name;
                    ss >> name;
                    mat->medium = find_or_add_med(meds, name);
                } else if (key == "mirror") {
                    read3(ss, mat->mirror);
                } else if (key == "ior") {
                    ss >> mat->ior;
                } else if (key == "priority") {
                    ss >> mat->priority;
                } else if (key == "geometryType") {
                    std::string g;
                    ss >> g;
                    if (!g.empty() && g[0] == 'r') mat->real = true;
                    else if (!g.empty() && g[0] == 'i') mat->real = false;
                    else {
                        set_error("unknown geometry type");
                        return UPBP_ERR_SCENE;
                    }
                } else if (key == "Ke") {
                    read3(ss, mat->ke);
                    mat->emissive = mat->ke[0] > 0.f || mat->ke[1] > 0.f || mat->ke[2] > 0.f;
                } else {
                    std::string name;
                    ss >> name;
                    const int m = find_mat(mats, name);
                    if (m < 0) {
                        set_error("material not found: " + name);
                        return UPBP_ERR_SCENE;
                    }
                    mat->enclosing = m;
                }
            } else if (key == "g" || key == "absorption" || key == "scattering" || key == "emission" ||
                       key == "continuation_probability") {
                if (med < 0) {
                    set_error("using " + key + " option without medium selection");
                    return UPBP_ERR_SCENE;
                }
                ObjMed& m = meds[med];
                if (key == "g") ss >> m.g;
                else if (key == "absorption") read3(ss, m.absorption);
                else if (key == "scattering") read3(ss, m.scattering);
                else if (key == "emission") read3(ss, m.emission);
                else ss >> m.cont;
            } else if (key == "globalMediumId") {
                std::string name;
                ss >> name;
                global_med = find_or_add_med(meds, name);
            } else if (key == "light_point" || key == "light_directional") {
                AuxLight l;
                l.type = key == "light_point" ? UPBP_LIGHT_POINT : UPBP_LIGHT_DIRECTIONAL;
                read3(ss, l.pos);
                read3(ss, l.emission);
                aux_lights.push_back(l);
            } else if (key == "light_background_constant") {
                AuxLight l;
                l.type = UPBP_LIGHT_BACKGROUND;
                read3(ss, l.emission);
                aux_lights.push_back(l);
            } else if (key == "light_background_em") {
                // light_background_em <scale> <rotate> <file> (scene_loader_obj.cpp:582-591);
                // a relative file name is relative to the OBJ file
                AuxLight l;
                l.type = UPBP_LIGHT_BACKGROUND;
                std::string file;
                if (!(ss >> l.env_scale >> l.env_rotate >> file)) {
                    set_error("light_background_em needs <scale> <rotate> <file>");
                    return UPBP_ERR_SCENE;
                }
                l.env_map = (file.size() > 1 && (file[1] == ':' || file[0] == '/')) ? file : dir_of(path) + file;
                aux_lights.push_back(l);
            }
        }

        upbp_scene* sc = new upbp_scene();
        sc->desc.background_light = -1;
        // lights from the AUX file first
        for (const AuxLight& al : aux_lights) {
            upbp_light L{};
            L.type = al.type;
            L.mat_id = L.med_id = -1;
            L.scale = 1.f;
            std::memcpy(L.intensity, al.emission, sizeof(L.intensity));
            std::memcpy(L.position, al.pos, sizeof(L.position));
            if (al.type == UPBP_LIGHT_BACKGROUND) {
                if (sc->desc.background_light < 0) {
                    sc->desc.background_light = (int32_t)sc->lights.size();
                    if (!al.env_map.empty()) {
                        const int rc = load_env_map(al.env_map, al.env_rotate, al.env_scale, *sc);
                        if (rc != UPBP_OK) {
                            delete sc;
                            return rc;
                        }
                    }
                }
            }
            sc->lights.push_back(L);
        }
        // triangles (file order), one area light per emissive triangle
        const size_t nt = tris.size();
        sc->verts.resize(9 * nt);
        sc->normals.resize(12 * nt);
        sc->tri_material.resize(nt);
        sc->tri_light.resize(nt);
        float bmin[3] = {1e36f, 1e36f, 1e36f}, bmax[3] = {-1e36f, -1e36f, -1e36f};
        for (size_t k = 0; k < nt; k++) {
            const Tri& t = tris[k];
            F3 p[3];
            for (int j = 0; j < 3; j++) {
                const int vi = t.v[j];
                if (vi < 0 || 3 * (size_t)vi + 2 >= v.size()) {
                    delete sc;
                    set_error("face references a missing vertex");
                    return UPBP_ERR_SCENE;
                }
                p[j] = {v[3 * vi], v[3 * vi + 1], v[3 * vi + 2]};
                sc->verts[9 * k + 3 * j + 0] = p[j].x;
                sc->verts[9 * k + 3 * j + 1] = p[j].y;
                sc->verts[9 * k + 3 * j + 2] = p[j].z;
                const float* q = &p[j].x;
                for (int a = 0; a < 3; a++) {
                    bmin[a] = std::fmin(bmin[a], q[a]);
                    bmax[a] = std::fmax(bmax[a], q[a]);
                }
            }
            F3 face = fnormalize(fcross(fsub(p[1], p[0]), fsub(p[2], p[0])));
            F3 n[3];
            if (t.n[0] >= 0 && t.n[1] >= 0 && t.n[2] >= 0) {
                for (int j = 0; j < 3; j++) {
                    const int ni = t.n[j];
                    if (3 * (size_t)ni + 2 >= vn.size()) {
                        delete sc;
                        set_error("face references a missing normal");
                        return UPBP_ERR_SCENE;
                    }
                    n[j] = {vn[3 * ni], vn[3 * ni + 1], vn[3 * ni + 2]};
                }
                const F3 mdl{(n[0].x + n[1].x + n[2].x) / 3.f, (n[0].y + n[1].y + n[2].y) / 3.f,
                             (n[0].z + n[1].z + n[2].z) / 3.f};
                if (fdot(face, mdl) < 0.f) face = fneg(face);
            } else {
                n[0] = n[1] = n[2] = face;
            }
            for (int j = 0; j < 3; j++) {
                sc->normals[12 * k + 3 * j + 0] = n[j].x;
                sc->normals[12 * k + 3 * j + 1] = n[j].y;
                sc->normals[12 * k + 3 * j + 2] = n[j].z;
            }
            sc->normals[12 * k + 9] = face.x;
            sc->normals[12 * k + 10] = face.y;
            sc->normals[12 * k + 11] = face.z;
            sc->tri_material[k] = t.mat;
            sc->tri_light[k] = -1;
            const ObjMat& m = mats[t.mat];
            if (m.emissive) {
                upbp_light L{};
                L.type = UPBP_LIGHT_AREA;
                L.mat_id = m.enclosing < 0 ? -1 : m.enclosing;
                L.med_id = L.mat_id < 0 ? -1 : mats[L.mat_id].medium;
                for (int a = 0; a < 3; a++) {
                    L.p0[a] = (&p[0].x)[a];
                    L.p1[a] = (&p[1].x)[a];
                    L.p2[a] = (&p[2].x)[a];
                    L.intensity[a] = m.ke[a];
                }
                L.scale = 1.f;
                sc->tri_light[k] = (int32_t)sc->lights.size();
                sc->lights.push_back(L);
            }
        }
        // materials
        for (const ObjMat& m : mats) {
            upbp_material M{};
            std::memcpy(M.diffuse, m.kd, sizeof(M.diffuse));
            std::memcpy(M.phong, m.ks, sizeof(M.phong));
            std::memcpy(M.mirror, m.mirror, sizeof(M.mirror));
            M.ior = m.ior;
            M.phong_exponent = m.ns;
            M.priority = m.priority;
            M.real = m.real ? 1 : 0;
            if (m.ns == 0.f) M.phong[0] = M.phong[1] = M.phong[2] = 0.f;
            M.medium = m.medium;
            sc->materials.push_back(M);
        }
        // media; continuation probability from albedo unless given
        for (const ObjMed& m : meds) {
            upbp_medium M{};
            std::memcpy(M.absorption, m.absorption, sizeof(M.absorption));
            std::memcpy(M.emission, m.emission, sizeof(M.emission));
            std::memcpy(M.scattering, m.scattering, sizeof(M.scattering));
            M.mean_cosine = m.g;
            float cp = m.cont;
            if (cp == -1.f) {
                float al[3];
                for (int a = 0; a < 3; a++) al[a] = m.scattering[a] / (m.scattering[a] + m.absorption[a]);
                const float mx = std::fmax(al[0], std::fmax(al[1], al[2]));
                if (std::isnan(mx) || std::isinf(mx)) cp = 1.f;
                else cp = mx > .8f ? mx : .8f;
            }
            M.continuation_prob = cp;
            sc->media.push_back(M);
        }
        if (global_med < 0) {
            upbp_medium M{};
            M.continuation_prob = 1.f;
            sc->media.push_back(M);
            sc->desc.global_medium = (int32_t)sc->media.size() - 1;
        } else {
            sc->desc.global_medium = global_med;
        }
        // camera (rows: right, up, -forward, position; fill_camera_info)
        upbp_camera_desc& cd = sc->desc.camera;
        for (int a = 0; a < 3; a++) {
            cd.origin[a] = tm[3][a];
            cd.target[a] = tm[3][a] - tm[2][a];
            cd.roll[a] = tm[1][a];
        }
        const float rl = 1.f / std::sqrt(cd.roll[0] * cd.roll[0] + cd.roll[1] * cd.roll[1] + cd.roll[2] * cd.roll[2]);
        for (int a = 0; a < 3; a++) cd.roll[a] *= rl;
        cd.horizontal_fov_deg = fov_rad * 57.295779f;
        cd.focal_dist = focal;
        cd.mat_id = cam_mat < 0 ? -1 : cam_mat;
        cd.med_id = cd.mat_id < 0 ? -1 : mats[cd.mat_id].medium;
        sc->desc.res_x = res_x;
        sc->desc.res_y = res_y;
        for (int a = 0; a < 3; a++) {
            sc->desc.bbox_min[a] = bmin[a];
            sc->desc.bbox_max[a] = bmax[a];
        }
        sc->finalize();
        *out = sc;
        return UPBP_OK;
    });
}

extern "C" int upbp_scene_load_predefined(int scene_id, uint32_t res_x, uint32_t res_y, upbp_scene** out)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!out || res_x == 0 || res_y == 0) return UPBP_ERR_ARGS;
        upbp_scene* sc = new upbp_scene();
        const int rc = build_predefined(scene_id, res_x, res_y, *sc);
        if (rc != UPBP_OK) {
            delete sc;
            return rc;
        }
        *out = sc;
        return UPBP_OK;
    });
}

extern "C" const upbp_scene_desc* upbp_scene_get_desc(const upbp_scene* scene) { return scene ? &scene->desc : nullptr; }

extern "C" void upbp_scene_free(upbp_scene* scene) { delete scene; }

extern "C" const char* upbp_last_error(void) { return get_error(); }
