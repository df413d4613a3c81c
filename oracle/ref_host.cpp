// Oracle translation unit 2: the reference's own command-line parser and scene
// loaders, compiled in place from the reference sources (never copied) and
// exposed through oracle_parse_and_load.  Test infrastructure only.
#include "misc/config.cpp"
#include "misc/scene_loader_obj.cpp"
#include "misc/scene_loader_predef.cpp"
#include "misc/tinyexr_wrapper.cpp"

#include "ref_setup.h"

#include <cstring>

int oracle_parse_and_load(int argc, const char** argv, OracleSetup* out)
{
    Config config{};
    int rc = parse_commandline(argc, argv, config);
    if (rc != 0) return rc;
    SceneLoader* loader = new SceneLoader{};
    loader->load_scene(config);
    out->scene = loader->scene;
    out->records = loader->records;
    out->record_count = loader->record_count;
    out->algorithm_flags = config.algorithm_flags;
    out->iteration_count = config.iteration_count;
    out->res_x = config.resolution.x;
    out->res_y = config.resolution.y;
    out->max_path_length = config.max_path_length;
    out->min_path_length = config.min_path_length;
    out->path_count_per_iter = config.path_count_per_iter;
    out->query_beam_type = (int)config.query_beam_type;
    out->photon_beam_type = (int)config.photon_beam_type;
    out->bb1d_radius_initial = config.bb1d_radius_initial;
    out->bb1d_radius_alpha = config.bb1d_radius_alpha;
    out->bb1d_used_light_subpath_count = config.bb1d_used_light_subpath_count;
    out->bp2d_radius_initial = config.bp2d_radius_initial;
    out->bp2d_radius_alpha = config.bp2d_radius_alpha;
    out->pb2d_radius_initial = config.pb2d_radius_initial;
    out->pb2d_radius_alpha = config.pb2d_radius_alpha;
    out->pp3d_radius_initial = config.pp3d_radius_initial;
    out->pp3d_radius_alpha = config.pp3d_radius_alpha;
    out->surf_radius_initial = config.surf_radius_initial;
    out->surf_radius_alpha = config.surf_radius_alpha;
    out->ignore_fully_spec_paths = config.ignore_fully_spec_paths;
    out->iteration_offset = config.iteration_offset;
    out->use_shading_normal = config.use_shading_normal;
    std::strncpy(out->output_name, config.output_name.c_str(), sizeof(out->output_name) - 1);
    out->output_name[sizeof(out->output_name) - 1] = 0;
    delete loader;  // the Scene arrays stay alive; they are owned by *out now
    return 0;
}

void oracle_free_setup(OracleSetup* s)
{
    delete_scene_host(s->scene);
    free(s->records);
}

// Writes an RGB float image (rows top to bottom) with tinyexr's own encoder:
// channels B, G, R stored as HALF (half != 0) or FLOAT with the given
// compression (0 none, 1 RLE, 2 ZIPS, 3 ZIP).  Makes test files for the
// library's EXR reader.  Returns tinyexr's status (0 on success).
extern "C" int upbp_ref_save_exr(const char* path, const float* rgb, int w, int h, int half, int compression)
{
    std::vector<float> ch[3];
    for (int k = 0; k < 3; k++) ch[k].resize((size_t)w * h);
    for (size_t i = 0; i < (size_t)w * h; i++)
        for (int k = 0; k < 3; k++) ch[k][i] = rgb[3 * i + k];
    EXRHeader header;
    InitEXRHeader(&header);
    EXRImage image;
    InitEXRImage(&image);
    float* planes[3] = {ch[2].data(), ch[1].data(), ch[0].data()};  // B, G, R
    image.images = reinterpret_cast<unsigned char**>(planes);
    image.num_channels = 3;
    image.width = w;
    image.height = h;
    EXRChannelInfo infos[3];
    std::memset(infos, 0, sizeof(infos));
    const char* names[3] = {"B", "G", "R"};
    int types[3], requested[3];
    for (int k = 0; k < 3; k++) {
        std::strncpy(infos[k].name, names[k], 255);
        types[k] = TINYEXR_PIXELTYPE_FLOAT;
        requested[k] = half ? TINYEXR_PIXELTYPE_HALF : TINYEXR_PIXELTYPE_FLOAT;
    }
    header.num_channels = 3;
    header.channels = infos;
    header.pixel_types = types;
    header.requested_pixel_types = requested;
    header.compression_type = compression;
    const char* err = nullptr;
    const int ret = SaveEXRImageToFile(&image, &header, path, &err);
    if (err) FreeEXRErrorMessage(err);
    return ret;
}
