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
