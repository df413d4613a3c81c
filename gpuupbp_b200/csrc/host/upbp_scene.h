// Host-side scene owned by the library (the result of the OBJ/AUX loader) and
// the camera set-up shared by the loader and the device context.
#pragma once

#include <exception>
#include <new>
#include <string>
#include <vector>

#include "../../../include/upbp.h"

struct upbp_scene {
    std::vector<float> verts, normals;
    std::vector<int32_t> tri_material, tri_light;
    std::vector<float> spheres;  // centre xyz, radius
    std::vector<float> env_rgb;  // environment map of the background light
    uint32_t env_width = 0, env_height = 0;
    std::vector<int32_t> sph_material;
    std::vector<upbp_material> materials;
    std::vector<upbp_medium> media;
    std::vector<upbp_light> lights;
    upbp_scene_desc desc{};
    void finalize();  // points desc at the vectors
};

namespace upbp_host {

// Camera matrices and image-plane distance (gpuupbp/host/camera.hpp:33-76),
// row-major 4x4.
struct CameraMatrices {
    float origin[3], direction[3];
    float raster_to_world[16], world_to_raster[16];
    float image_plane_dist;
};
CameraMatrices camera_setup(const upbp_camera_desc& c, float res_x, float res_y);

void set_error(const std::string& msg);

// OpenEXR scanline image (NONE/RLE/ZIPS/ZIP, HALF/FLOAT) as RGB floats.
bool read_exr_rgb(const std::string& path, int& width, int& height, std::vector<float>& rgb, std::string& err);
int load_env_map(const std::string& path, float rotate, float scale, upbp_scene& sc);

// The reference's predefined Cornell-box scenes (-s 0..40).
int predefined_scene_count();
const char* predefined_scene_name(int id, bool long_name);
int build_predefined(int id, uint32_t res_x, uint32_t res_y, upbp_scene& sc);

// Runs the body of a C entry point and turns a C++ exception (a failed host
// allocation, a thread that could not start) into UPBP_ERR_HOST with its
// message: no exception crosses the C ABI.
template <class F>
int abi_guard(F&& body) noexcept
{
    try {
        return body();
    } catch (const std::bad_alloc&) {
        set_error("out of host memory");
    } catch (const std::exception& e) {
        try {
            set_error(std::string("host error: ") + e.what());
        } catch (...) {
        }
    } catch (...) {
    }
    return UPBP_ERR_HOST;
}

}  // namespace upbp_host
