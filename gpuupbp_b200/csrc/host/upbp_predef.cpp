// The 41 predefined Cornell-box scenes (-s 0..40): the reference's scene table
// (gpuupbp/misc/config.cpp:100-548, types in misc/scene_config.hpp:32-110) and
// its construction of geometry, materials, media, lights and camera
// (gpuupbp/misc/scene_loader_predef.cpp:126-603).  The table, the constants
// and the material-sharing rule are the reference's, so that a scene id
// names the same scene in both programs; the order of operations in the
// float arithmetic follows the reference so the records agree bit for bit.
#include <cmath>
#include <cstring>
#include <vector>

#include "upbp_scene.h"

namespace upbp_host {
namespace {

// scene_config.hpp:46-61
enum Geom : int { kLeftWall, kRightWall, kFrontWallFacing, kFrontWallBack, kBackWall, kCeiling, kFloor,
                  kSphLarge, kSphLeft, kSphRight, kSphBottomLeft, kSphBottomRight, kSphTop, kSphVeryLarge,
                  kBoxVeryLarge, kGeomCount };
// scene_config.hpp:63-75 (kNone: imaginary element)
enum Mat : int { kNone = -1, kWaterMat, kIce, kGlass, kRed, kGreen, kBlue, kWhite, kGlossy, kMirror, kLightMat,
                 kBaseMats };
// scene_config.hpp:77-93 (kNoMed: no medium)
enum Med : int { kNoMed = -1, kClear, kWaterMed, kIso, kAniso, kWeakIso, kWeakYellowIso, kWeakAniso, kRedAbs,
                 kYellowEmit, kYellowGreen, kBlueAbsEmit, kReddish, kAbsAniso, kMediaCount };
// scene_config.hpp:34-44
enum Light : int { kCeilBig, kCeilSmall, kCeilSmallDistant, kCeilPoint, kFacingSmall, kFacingPoint, kSun,
                   kBackground, kNoLight };
// the Cornell boxes the table starts from (config.cpp:107-128)
enum Box : int { kNoBox, kDiffuseFloor, kGlossyFloor, kWhiteBack };

struct Element {
    Geom g;
    Mat m;
    Med d;
};

struct SceneDef {
    const char* short_name;
    const char* long_name;
    Light light;
    Med global;
    Box box;
    std::vector<Element> extra;
};

const Element kGlassBL{kSphBottomLeft, kGlass, kNoMed};
const Element kWaterBR{kSphBottomRight, kWaterMat, kWaterMed};
const Element kIceTop{kSphTop, kIce, kNoMed};

const std::vector<SceneDef>& table()
{
    static const std::vector<SceneDef> t = {
        {"abssph", "large absorbing sphere + big area light", kCeilBig, kClear, kDiffuseFloor,
         {{kSphLarge, kNone, kRedAbs}}},
        {"isosph", "large isoscattering sphere + small area light", kCeilSmall, kClear, kDiffuseFloor,
         {{kSphLarge, kNone, kIso}}},
        {"mirsphinfisov", "large mirror sphere + weak isoscattering + small area light", kCeilSmall, kWeakIso,
         kGlossyFloor, {{kSphLarge, kMirror, kNoMed}}},
        {"smswiso", "small media spheres + weak isoscattering + small area light", kCeilSmall, kWeakIso,
         kDiffuseFloor, {{kSphLeft, kNone, kBlueAbsEmit}, {kSphRight, kNone, kYellowGreen}}},
        {"smswani", "small media spheres + weak anisoscattering + small area light", kCeilSmall, kWeakAniso,
         kDiffuseFloor, {{kSphLeft, kNone, kBlueAbsEmit}, {kSphRight, kNone, kYellowGreen}}},
        {"ssssun", "specular small spheres + sun", kSun, kClear, kGlossyFloor,
         {{kSphLeft, kMirror, kNoMed}, {kSphRight, kGlass, kNoMed}}},
        {"ssspoint", "specular small spheres + point light", kCeilPoint, kClear, kGlossyFloor,
         {{kSphLeft, kMirror, kNoMed}, {kSphRight, kGlass, kNoMed}}},
        {"sssback", "specular small spheres + background light", kBackground, kClear, kGlossyFloor,
         {{kSphLeft, kMirror, kNoMed}, {kSphRight, kGlass, kNoMed}}},
        {"mirsph", "large mirror sphere + small area light", kCeilSmall, kClear, kGlossyFloor,
         {{kSphLarge, kMirror, kNoMed}}},
        {"emisph", "large emitting sphere + small area light", kCeilSmall, kClear, kDiffuseFloor,
         {{kSphLarge, kNone, kYellowEmit}}},
        {"gemisph", "large glass emitting sphere", kNoLight, kClear, kDiffuseFloor,
         {{kSphLarge, kGlass, kYellowEmit}}},
        {"nogeoisobig", "no geometry + isoscattering + big area light", kCeilBig, kIso, kNoBox, {}},
        {"nogeoisosmall", "no geometry + isoscattering + small area light", kCeilSmall, kIso, kNoBox, {}},
        {"nogeoisopt", "no geometry + isoscattering + point light", kCeilPoint, kIso, kNoBox, {}},
        {"nogeoanibig", "no geometry + anisoscattering + big area light", kCeilBig, kAniso, kNoBox, {}},
        {"nogeoanismall", "no geometry + anisoscattering + small area light", kCeilSmall, kAniso, kNoBox, {}},
        {"nogeoanipt", "no geometry + anisoscattering + point light", kCeilPoint, kAniso, kNoBox, {}},
        {"faceisosmall", "no geometry + isoscattering + facing small area light", kFacingSmall, kIso, kNoBox, {}},
        {"faceisopt", "no geometry + isoscattering + facing point light", kFacingPoint, kIso, kNoBox, {}},
        {"faceanismall", "no geometry + anisoscattering + facing small area light", kFacingSmall, kAniso, kNoBox,
         {}},
        {"faceanipt", "no geometry + anisoscattering + facing point light", kFacingPoint, kAniso, kNoBox, {}},
        {"overgwi", "three overlapping spheres (glass, water, ice) + big area light", kCeilBig, kClear, kWhiteBack,
         {kGlassBL, kWaterBR, kIceTop}},
        {"rovergwi", "three overlapping spheres (glass, water, ice) + one big red sphere + big area light", kCeilBig,
         kClear, kWhiteBack, {kGlassBL, kWaterBR, kIceTop, {kSphVeryLarge, kNone, kRedAbs}}},
        {"wovergwi", "three overlapping spheres (glass, water, ice) + one big water sphere + big area light",
         kCeilBig, kClear, kWhiteBack, {kGlassBL, kWaterBR, kIceTop, {kSphVeryLarge, kWaterMat, kWaterMed}}},
        {"iovergwi", "three overlapping spheres (glass, water, ice) + one big ice sphere + big area light", kCeilBig,
         kClear, kWhiteBack, {kGlassBL, kWaterBR, kIceTop, {kSphVeryLarge, kIce, kNoMed}}},
        {"govergwi", "three overlapping spheres (glass, water, ice) + one big glass sphere + big area light",
         kCeilBig, kClear, kWhiteBack, {kGlassBL, kWaterBR, kIceTop, {kSphVeryLarge, kGlass, kNoMed}}},
        {"movergwi", "three overlapping spheres (glass, water, ice) + one big mirror sphere + big area light",
         kCeilBig, kClear, kWhiteBack, {kGlassBL, kWaterBR, kIceTop, {kSphVeryLarge, kMirror, kNoMed}}},
        {"aniovergwi", "three overlapping spheres (glass, water, ice) + weak anisoscattering + small area light",
         kCeilSmall, kWeakAniso, kWhiteBack, {kGlassBL, kWaterBR, kIceTop}},
        {"overiwr", "three overlapping glass spheres (iso, water, red absorb) + big area light", kCeilBig, kClear,
         kWhiteBack,
         {{kSphBottomLeft, kGlass, kIso}, {kSphBottomRight, kGlass, kWaterMed}, {kSphTop, kGlass, kRedAbs}}},
        {"isooveriwr", "three overlapping spheres (iso, water, red absorb) + weak isoscattering + big area light",
         kCeilBig, kWeakIso, kNoBox,
         {{kSphBottomLeft, kNone, kIso}, {kSphBottomRight, kNone, kWaterMed}, {kSphTop, kNone, kRedAbs}}},
        {"woveriwr",
         "three overlapping spheres (iso, water, red absorb) + one big water sphere + background light",
         kBackground, kClear, kWhiteBack,
         {{kSphBottomLeft, kNone, kIso},
          {kSphBottomRight, kNone, kWaterMed},
          {kSphTop, kNone, kRedAbs},
          {kSphVeryLarge, kNone, kWaterMed}}},
        {"backg", "only background light and global medium", kBackground, kReddish, kNoBox, {}},
        {"backas", "only background light and absorbing sphere", kBackground, kClear, kNoBox,
         {{kSphVeryLarge, kNone, kRedAbs}}},
        {"backss", "only background light and scattering sphere", kBackground, kClear, kNoBox,
         {{kSphVeryLarge, kNone, kIso}}},
        {"bigss", "only big area light and scattering sphere", kCeilBig, kClear, kNoBox,
         {{kSphVeryLarge, kNone, kIso}}},
        {"smallsb", "only small area light and scattering box", kCeilSmallDistant, kClear, kNoBox,
         {{kBoxVeryLarge, kNone, kWeakYellowIso}}},
        {"ssssuninfisov", "specular small spheres + weak anisoscattering + sun", kSun, kWeakIso, kGlossyFloor,
         {{kSphLeft, kMirror, kNoMed}, {kSphRight, kGlass, kNoMed}}},
        {"ssspointinfisov", "specular small spheres + weak anisoscattering + point light", kCeilPoint, kWeakIso,
         kGlossyFloor, {{kSphLeft, kMirror, kNoMed}, {kSphRight, kGlass, kNoMed}}},
        {"sssbackinfisov", "specular small spheres + weak anisoscattering + background light", kBackground,
         kWeakIso, kGlossyFloor, {{kSphLeft, kMirror, kNoMed}, {kSphRight, kGlass, kNoMed}}},
        {"glasssphbck", "large glass medium sphere + background light", kBackground, kClear, kGlossyFloor,
         {{kSphLarge, kGlass, kAbsAniso}}},
        {"glasssphbck", "large glass medium sphere + large area light", kCeilBig, kClear, kGlossyFloor,
         {{kSphLarge, kGlass, kAbsAniso}}},
    };
    return t;
}

// The element list of a scene: its Cornell box, then its own elements.
std::vector<Element> elements_of(const SceneDef& s)
{
    std::vector<Element> e;
    if (s.box != kNoBox) {
        e.push_back({kLeftWall, kGreen, kNoMed});
        e.push_back({kRightWall, kRed, kNoMed});
        e.push_back({kBackWall, s.box == kWhiteBack ? kWhite : kBlue, kNoMed});
        e.push_back({kCeiling, kWhite, kNoMed});
        e.push_back({kFloor, s.box == kGlossyFloor ? kGlossy : kWhite, kNoMed});
    }
    e.insert(e.end(), s.extra.begin(), s.extra.end());
    return e;
}

struct P3 {
    float x, y, z;
};
P3 operator+(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
P3 operator-(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
P3 operator*(P3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
P3 cross3(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
P3 unit(P3 a)
{
    const float inv = 1.f / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return a * inv;
}
void put(float* d, P3 p)
{
    d[0] = p.x;
    d[1] = p.y;
    d[2] = p.z;
}

struct Tri {
    P3 p[3];
    int mat, light;
};
struct Sph {
    P3 c;
    float r;
    int mat;
};

upbp_material base_material()  // reset_material (host/material.hpp:32-41) on a zeroed record
{
    upbp_material m{};
    m.phong_exponent = 1.f;
    m.ior = -1.f;
    m.priority = -1;  // thin wall
    m.real = 1;
    m.medium = 0;     // reset_material leaves the medium index as it was: zero
    return m;
}

upbp_medium medium(P3 a, P3 e, P3 s, float cont = .8f, float g = 0.f)
{
    upbp_medium m{};
    put(m.absorption, a);
    put(m.emission, e);
    put(m.scattering, s);
    m.continuation_prob = cont;
    m.mean_cosine = g;
    return m;
}

}  // namespace

int predefined_scene_count() { return (int)table().size(); }

const char* predefined_scene_name(int id, bool long_name)
{
    if (id < 0 || id >= predefined_scene_count()) return nullptr;
    return long_name ? table()[id].long_name : table()[id].short_name;
}

int build_predefined(int id, uint32_t res_x, uint32_t res_y, upbp_scene& sc)
{
    if (id < 0 || id >= predefined_scene_count()) {
        set_error("predefined scene id out of range 0..40");
        return UPBP_ERR_ARGS;
    }
    const SceneDef& def = table()[id];
    auto rgb = [](float r, float g, float b) { return P3{r, g, b}; };

    // materials (scene_loader_predef.cpp:140-196)
    std::vector<upbp_material> mats(kBaseMats, base_material());
    put(mats[kRed].diffuse, rgb(0.803922f, 0.152941f, 0.152941f));
    put(mats[kGreen].diffuse, rgb(0.156863f, 0.803922f, 0.172549f));
    put(mats[kBlue].diffuse, rgb(0.156863f, 0.172549f, 0.803922f));
    put(mats[kWhite].diffuse, rgb(0.803922f, 0.803922f, 0.803922f));
    put(mats[kGlossy].diffuse, rgb(.1f, .1f, .1f));
    put(mats[kGlossy].phong, rgb(.7f, .7f, .7f));
    mats[kGlossy].phong_exponent = 90.f;
    put(mats[kMirror].mirror, rgb(1.f, 1.f, 1.f));
    put(mats[kWaterMat].mirror, rgb(.7f, .7f, .7f));
    mats[kWaterMat].ior = 1.33f;
    put(mats[kIce].mirror, rgb(.5f, .5f, .5f));
    mats[kIce].ior = 1.31f;
    put(mats[kGlass].mirror, rgb(1.f, 1.f, 1.f));
    mats[kGlass].ior = 1.6f;

    // media (scene_loader_predef.cpp:198-290); continuation probability 0.8
    // except the clear medium (init_medium_clear: 1)
    const P3 z{0.f, 0.f, 0.f};
    sc.media.assign(kMediaCount, upbp_medium{});
    sc.media[kClear] = medium(z, z, z, 1.f);
    sc.media[kWaterMed] = medium(rgb(.7f, .6f, 0.f), z, z);
    sc.media[kRedAbs] = medium(rgb(0.f, 1.f, 1.f), z, z);
    sc.media[kYellowEmit] = medium(z, rgb(.7f, .7f, 0.f), z);
    sc.media[kYellowGreen] = medium(rgb(.5f, 0.f, .5f), rgb(1.f, 1.f, 0.f), rgb(.1f, .1f, 0.f));
    sc.media[kBlueAbsEmit] = medium(rgb(.1f, .1f, 0.f), rgb(0.f, 0.f, 1.f), z);
    sc.media[kIso] = medium(z, z, rgb(.9f, .9f, .9f));
    sc.media[kAniso] = medium(z, z, rgb(.9f, .9f, .9f), .8f, .6f);
    sc.media[kWeakIso] = medium(z, z, rgb(.1f, .1f, .1f));
    sc.media[kWeakYellowIso] = medium(z, z, rgb(.1f, .1f, 0.f));
    sc.media[kWeakAniso] = medium(z, z, rgb(.1f, .1f, .1f), .8f, .6f);
    sc.media[kReddish] = medium(rgb(0.f, .02f, 0.f), z, rgb(.002f, .002f, 0.f), .8f, .6f);
    sc.media[kAbsAniso] = medium(rgb(.02f, 2.f, 2.f), z, rgb(12.f, 20.f, 20.f), .8f, -.3f);
    sc.desc.global_medium = def.global;

    // geometry (scene_loader_predef.cpp:292-444)
    const P3 cb[8] = {{-1.27029f, 1.30455f, -1.28002f}, {1.28975f, 1.30455f, -1.28002f},
                      {1.28975f, 1.30455f, 1.28002f},   {-1.27029f, 1.30455f, 1.28002f},
                      {-1.27029f, -1.25549f, -1.28002f}, {1.28975f, -1.25549f, -1.28002f},
                      {1.28975f, -1.25549f, 1.28002f},   {-1.27029f, -1.25549f, 1.28002f}};
    const P3 floor_c = (cb[0] + cb[1] + cb[4] + cb[5]) * (1.f / 4.f);
    const P3 box_c = (cb[0] + cb[1] + cb[2] + cb[3] + cb[4] + cb[5] + cb[6] + cb[7]) * (1.f / 8.f);
    const float r_large = .8f, r_small = .5f, r_very_large = 1.f;
    const P3 c_large = floor_c + P3{0.f, 0.f, r_large + .01f};
    const P3 left_wall_c = (cb[0] + cb[4]) * (1.f / 2.f) + P3{0.f, 0.f, r_small + .01f};
    const P3 right_wall_c = (cb[1] + cb[5]) * (1.f / 2.f) + P3{0.f, 0.f, r_small + .01f};
    const float xlen = right_wall_c.x - left_wall_c.x;
    const P3 c_left = left_wall_c + P3{2.f * xlen / 7.f, 0.f, 0.f};
    const P3 c_right = right_wall_c - P3{2.f * xlen / 7.f, 0.f, 0.f};
    const float ov = .5f * r_small;
    const P3 c_bl = box_c + P3{-ov, 0.f, -ov}, c_br = box_c + P3{ov, 0.f, -ov}, c_top = box_c + P3{0.f, 0.f, ov};

    std::vector<Tri> tris[2];  // [0] real, [1] imaginary
    std::vector<Sph> sphs[2];
    bool used[kGeomCount] = {};
    for (const Element& e : elements_of(def)) {
        if (used[e.g]) continue;
        used[e.g] = true;
        const int cls = e.m >= 0 ? 0 : 1;
        // a sphere or the large box gets its own material with the priority
        // rule of the SmallUPBP thesis, shared by elements of equal priority;
        // walls use the base material
        int mat_id = e.m;
        if (e.g > kFloor) {
            const int priority = (1 + e.m) * 10 + 1 + e.d;
            mat_id = kBaseMats;
            while (mat_id < (int)mats.size() && mats[mat_id].priority != priority) mat_id++;
            if (mat_id == (int)mats.size()) {
                upbp_material m = e.m >= 0 ? mats[e.m] : base_material();
                m.priority = priority;
                m.real = e.m >= 0 ? 1 : 0;
                mats.push_back(m);
            }
        }
        mats[mat_id].medium = e.d;
        auto tri = [&](P3 a, P3 b, P3 c) { tris[cls].push_back({{a, b, c}, mat_id, -1}); };
        auto sph = [&](P3 c, float r) { sphs[cls].push_back({c, r, mat_id}); };
        switch (e.g) {
        case kLeftWall: tri(cb[3], cb[7], cb[4]); tri(cb[4], cb[0], cb[3]); break;
        case kRightWall: tri(cb[1], cb[5], cb[6]); tri(cb[6], cb[2], cb[1]); break;
        case kFrontWallFacing: tri(cb[4], cb[5], cb[6]); tri(cb[6], cb[7], cb[4]); break;
        case kFrontWallBack: tri(cb[6], cb[5], cb[4]); tri(cb[4], cb[7], cb[6]); break;
        case kBackWall: tri(cb[0], cb[1], cb[2]); tri(cb[2], cb[3], cb[0]); break;
        case kCeiling:  // the big ceiling light replaces the ceiling
            if (def.light != kCeilBig) {
                tri(cb[2], cb[6], cb[7]);
                tri(cb[7], cb[3], cb[2]);
            }
            break;
        case kFloor: tri(cb[0], cb[4], cb[5]); tri(cb[5], cb[1], cb[0]); break;
        case kSphLarge: sph(c_large, r_large); break;
        case kSphLeft: sph(c_left, r_small); break;
        case kSphRight: sph(c_right, r_small); break;
        case kSphBottomLeft: sph(c_bl, r_small); break;
        case kSphBottomRight: sph(c_br, r_small); break;
        case kSphTop: sph(c_top, r_small); break;
        case kSphVeryLarge: sph(box_c, r_very_large); break;
        case kBoxVeryLarge:
            tri(cb[7], cb[3], cb[4]); tri(cb[0], cb[4], cb[3]); tri(cb[5], cb[1], cb[6]); tri(cb[2], cb[6], cb[1]);
            tri(cb[4], cb[5], cb[6]); tri(cb[6], cb[7], cb[4]); tri(cb[1], cb[0], cb[2]); tri(cb[3], cb[2], cb[0]);
            tri(cb[6], cb[2], cb[7]); tri(cb[3], cb[7], cb[2]); tri(cb[4], cb[0], cb[5]); tri(cb[1], cb[5], cb[0]);
            break;
        default: break;
        }
    }

    // lights (scene_loader_predef.cpp:446-545); area-light triangles are real
    // and come after the scene's geometry
    sc.desc.background_light = -1;
    auto new_light = [](int type) {
        upbp_light l{};
        l.type = type;
        l.mat_id = l.med_id = -1;
        l.scale = 1.f;
        return l;
    };
    auto area = [&](P3 a, P3 b, P3 c, float k) {
        upbp_light l = new_light(UPBP_LIGHT_AREA);
        put(l.p0, a);
        put(l.p1, b);
        put(l.p2, c);
        put(l.intensity, P3{k, k, k});
        tris[0].push_back({{a, b, c}, kLightMat, (int)sc.lights.size()});
        sc.lights.push_back(l);
    };
    auto point = [&](P3 pos) {
        const float k = 70.f * (0.318309886183790671538f * .25f);
        upbp_light l = new_light(UPBP_LIGHT_POINT);
        put(l.position, pos);
        put(l.intensity, P3{k, k, k});
        sc.lights.push_back(l);
    };
    auto small_box = [](float dy, P3* lb) {
        const float y0 = .25f + dy, y1 = -.25f + dy;
        const P3 v[8] = {{-.25f, y0, 1.26002f}, {.25f, y0, 1.26002f}, {.25f, y0, 1.28002f}, {-.25f, y0, 1.28002f},
                         {-.25f, y1, 1.26002f}, {.25f, y1, 1.26002f}, {.25f, y1, 1.28002f}, {-.25f, y1, 1.28002f}};
        for (int k = 0; k < 8; k++) lb[k] = v[k];
    };
    const float k_small = 25.03329895614464f;
    switch (def.light) {
    case kCeilBig:
        area(cb[2], cb[6], cb[7], 0.95492965f);
        area(cb[7], cb[3], cb[2], 0.95492965f);
        break;
    case kCeilSmall: {
        P3 lb[8];
        small_box(0.f, lb);
        // a white box around the light (back, left, right and front walls),
        // open at the bottom where the two light triangles are
        const int walls[8][3] = {{0, 2, 1}, {2, 0, 3}, {3, 4, 7}, {4, 3, 0}, {1, 6, 5}, {6, 1, 2}, {4, 5, 6}, {6, 7, 4}};
        for (const auto& w : walls) tris[0].push_back({{lb[w[0]], lb[w[1]], lb[w[2]]}, kWhite, -1});
        area(lb[0], lb[5], lb[4], k_small);
        area(lb[5], lb[0], lb[1], k_small);
        break;
    }
    case kCeilSmallDistant: {
        P3 lb[8];
        small_box(-1.5f, lb);
        area(lb[0], lb[5], lb[4], k_small);
        area(lb[5], lb[0], lb[1], k_small);
        break;
    }
    case kCeilPoint: point(P3{0.f, -.5f, 1.f}); break;
    case kFacingSmall: {
        const P3 lr[4] = {{-.25f, 0.f, .25f}, {.25f, 0.f, .25f}, {-.25f, 0.f, -.25f}, {.25f, 0.f, -.25f}};
        area(lr[2], lr[3], lr[0], k_small);
        area(lr[1], lr[0], lr[3], k_small);
        break;
    }
    case kFacingPoint: point(P3{0.f, 0.f, 0.f}); break;
    case kSun: {
        upbp_light l = new_light(UPBP_LIGHT_DIRECTIONAL);
        put(l.position, P3{-1.f, 1.5f, -1.f});  // the direction
        put(l.intensity, P3{.5f, .2f, 0.f} * 20.f);
        sc.lights.push_back(l);
        break;
    }
    case kBackground: {
        upbp_light l = new_light(UPBP_LIGHT_BACKGROUND);
        put(l.intensity, P3{135.f, 206.f, 250.f} * (1.f / 255.f));
        sc.desc.background_light = (int32_t)sc.lights.size();
        sc.lights.push_back(l);
        break;
    }
    case kNoLight: break;
    }

    // records: real triangles, real spheres, imaginary triangles, imaginary
    // spheres; the bounding box over all of them (set_triangles/set_spheres)
    float bmin[3] = {1e36f, 1e36f, 1e36f}, bmax[3] = {-1e36f, -1e36f, -1e36f};
    auto grow = [&](P3 p) {
        const float q[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; a++) {
            bmin[a] = std::fmin(bmin[a], q[a]);
            bmax[a] = std::fmax(bmax[a], q[a]);
        }
    };
    for (int cls = 0; cls < 2; cls++) {
        for (const Tri& t : tris[cls]) {
            const P3 n = unit(cross3(t.p[1] - t.p[0], t.p[2] - t.p[0]));
            for (int j = 0; j < 3; j++) {
                sc.verts.insert(sc.verts.end(), {t.p[j].x, t.p[j].y, t.p[j].z});
                grow(t.p[j]);
            }
            for (int j = 0; j < 4; j++) sc.normals.insert(sc.normals.end(), {n.x, n.y, n.z});
            sc.tri_material.push_back(t.mat);
            sc.tri_light.push_back(t.light);
        }
        for (const Sph& s : sphs[cls]) {
            sc.spheres.insert(sc.spheres.end(), {s.c.x, s.c.y, s.c.z, s.r});
            sc.sph_material.push_back(s.mat);
            grow(s.c - P3{s.r, s.r, s.r});
            grow(s.c + P3{s.r, s.r, s.r});
        }
    }
    sc.materials = mats;

    // camera (scene_loader_predef.cpp:130-137)
    upbp_camera_desc& cd = sc.desc.camera;
    put(cd.origin, P3{-0.0439815f, -4.12529f, 0.222539f});
    put(cd.target, P3{-0.03709525f, -3.126785f, 0.1683229f});
    put(cd.roll, P3{3.73896e-4f, 0.0542148f, 0.998529f});
    cd.horizontal_fov_deg = 45.f;
    cd.focal_dist = 1.f;
    cd.mat_id = cd.med_id = -1;
    sc.desc.res_x = res_x;
    sc.desc.res_y = res_y;
    for (int a = 0; a < 3; a++) {
        sc.desc.bbox_min[a] = bmin[a];
        sc.desc.bbox_max[a] = bmax[a];
    }
    sc.finalize();
    return UPBP_OK;
}

}  // namespace upbp_host
