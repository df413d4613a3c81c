// Plain record handed from the reference's own host code (command-line parser
// and scene loaders, compiled in oracle/ref_host.cpp) to the oracle driver
// (oracle/ref_driver.cpp).  Keeps the two translation units apart: the device
// sources and the host sources of the reference do not share one TU.
// Test infrastructure only.
#ifndef UPBP_ORACLE_REF_SETUP_H
#define UPBP_ORACLE_REF_SETUP_H

#include "shared/scene.h"

struct OracleSetup {
    Scene scene;           // filled by SceneLoader::load_scene (host pointers)
    Record* records;       // (material, light) pairs, one per SBT hit record
    unsigned int record_count;
    // Config fields the renderer reads (gpuupbp/misc/config.hpp:44-120)
    unsigned int algorithm_flags;
    int iteration_count;
    unsigned int res_x, res_y;
    unsigned int max_path_length;
    unsigned int min_path_length;
    float path_count_per_iter;
    int query_beam_type;
    int photon_beam_type;
    float bb1d_radius_initial, bb1d_radius_alpha, bb1d_used_light_subpath_count;
    float bp2d_radius_initial, bp2d_radius_alpha;
    float pb2d_radius_initial, pb2d_radius_alpha;
    float pp3d_radius_initial, pp3d_radius_alpha;
    float surf_radius_initial, surf_radius_alpha;
    bool ignore_fully_spec_paths;
    unsigned long long iteration_offset;
    bool use_shading_normal;
    char output_name[512];
};

// Runs the reference's parse_commandline and SceneLoader::load_scene.
// Returns 0 on success, 1 when the command line asked for help, -1 on a
// parse error (the reference prints the reason).
int oracle_parse_and_load(int argc, const char** argv, OracleSetup* out);
void oracle_free_setup(OracleSetup* s);

#endif
