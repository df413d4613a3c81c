// Command-line parser with the reference's flags, defaults and validation
// (gpuupbp/misc/config.cpp:735-1370), including the default output name
// (config.cpp:520-600).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "upbp_scene.h"

namespace {

void copy_str(char* dst, size_t cap, const std::string& s)
{
    std::strncpy(dst, s.c_str(), cap - 1);
    dst[cap - 1] = 0;
}

std::string two_digits(long v)
{
    char b[32];
    std::snprintf(b, sizeof(b), "%02ld", v);
    return b;
}

std::string default_suffix(const upbp_config& c, const std::string& extra)
{
    std::string s;
    if (c.iteration_count > 0) s += "_i" + two_digits(c.iteration_count);
    s += "_l" + two_digits(c.max_path_length);
    s += "_a";
    const uint32_t f = c.algorithm_flags;
    if (f & UPBP_BPT) s += "+bpt";
    if (f & UPBP_SURF) s += "+surf";
    if (f & UPBP_PP3D) s += "+pp3d";
    if (f & UPBP_PB2D) s += "+pb2d";
    if (f & UPBP_BB1D) s += "+bb1d";
    if (f & UPBP_BP2D) s += "+bp2d";
    if ((f & UPBP_PB2D) || (f & UPBP_BB1D)) s += std::string("_qbt") + (c.query_beam_type == UPBP_SHORT_BEAM ? "S" : "L");
    if ((f & UPBP_BP2D) || (f & UPBP_BB1D)) s += std::string("_pbt") + (c.photon_beam_type == UPBP_SHORT_BEAM ? "S" : "L");
    s += extra;
    s += ".exr";
    return s;
}

void print_usage(const char* prog)
{
    std::printf("\nUsage: %s [ -s <scene_id> | -a <algorithm> | -l <path length> |\n", prog);
    std::printf("           -t <time> | -i <iteration> | -o <output_name> ]\n\n");
    std::printf("    -s  <scene_id> selects the scene (default 0):\n");
    std::printf("        -1    <file.obj>: OBJ scene (with <file.obj>.aux)\n");
    for (int i = 0; i < upbp_host::predefined_scene_count(); i++)
        std::printf("        %-2d    %s\n", i, upbp_host::predefined_scene_name(i, true));
    std::printf("    -a  upbp_<tech>[+<tech>]* | upbp+<tech>... | upbp_all (tech=bpt|surf|pp3d|pb2d|bb1d|bp2d)\n");
    std::printf("    -l  maximum path length (default 10)   -i iterations (default 1)   -t seconds\n");
    std::printf("    -o  output name (.exr or .bmp)          -r WIDTHxHEIGHT (default 256x256)\n");
    std::printf("    -r_alpha[_surf|_pp3d|_pb2d|_bb1d|_bp2d] <a>  -r_initial[_...] <r> (negative: x scene radius)\n");
    std::printf("    -previous -compatible -speconly -ignorespec 0|1 -qbt S|L -pbt S|L -pbc <n>\n");
    std::printf("    -continuous_output <n> -pcpi <n> -sn 0|1 -assert -ioff <iter> -log\n");
    std::printf("    -guide <n>   (this build only) learned proposal for scattering in media, trained during\n"
                "                 the first n iterations\n");
    std::printf("    -mis_exact   (this build only) MIS weights of the full-path balance heuristic where the\n"
                "                 reference's recursion departs from it (photon-beam distances, NEE through media)\n");
    std::printf("    -checkpoint <file>  (this build only) write the render's state after the last iteration and\n"
                "                 at every continuous output;  -resume <file>  continue a render from one\n");
}

}  // namespace

extern "C" int upbp_parse_command_line(int argc, const char** argv, upbp_config* out)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!out) return UPBP_ERR_ARGS;
        upbp_config c{};
        c.scene_id = 0;
        c.algorithm_flags = UPBP_BPT | UPBP_SURF | UPBP_PP3D | UPBP_PB2D | UPBP_BB1D;
        c.iteration_count = 1;
        c.max_time = -1.f;
        c.res_x = c.res_y = 256;
        c.max_path_length = 10;
        c.min_path_length = 0;
        c.path_count_per_iter = -1.f;
        c.query_beam_type = UPBP_LONG_BEAM;
        c.photon_beam_type = UPBP_SHORT_BEAM;
        c.surf_radius_initial = -0.0015f;
        c.surf_radius_alpha = 0.75f;
        c.pp3d_radius_initial = c.pb2d_radius_initial = c.bb1d_radius_initial = c.bp2d_radius_initial = -0.001f;
        c.pp3d_radius_alpha = c.pb2d_radius_alpha = c.bb1d_radius_alpha = c.bp2d_radius_alpha = 1.f;
        c.bb1d_used_light_subpath_count = -1.f;
        c.use_shading_normal = 1;
        std::ostringstream extra;
        bool set_alpha[5] = {false, false, false, false, false};  // surf pp3d pb2d bb1d bp2d
        bool set_init[5] = {false, false, false, false, false};
        float* alphas[5] = {&c.surf_radius_alpha, &c.pp3d_radius_alpha, &c.pb2d_radius_alpha, &c.bb1d_radius_alpha,
                            &c.bp2d_radius_alpha};
        float* inits[5] = {&c.surf_radius_initial, &c.pp3d_radius_initial, &c.pb2d_radius_initial, &c.bb1d_radius_initial,
                           &c.bp2d_radius_initial};
        const char* tech_names[5] = {"surf", "pp3d", "pb2d", "bb1d", "bp2d"};

        auto fail = [&](const std::string& msg) {
            std::fprintf(stderr, "%s, please see help (-h)\n", msg.c_str());
            upbp_host::set_error(msg);
            return UPBP_ERR_ARGS;
        };

        for (int i = 1; i < argc; i++) {
            const std::string a = argv[i];
            if (a == "-h" || a == "--help" || a == "/?" || a == "-hf" || a == "--help_full" || a == "/??") {
                print_usage(argv[0]);
                return UPBP_HELP;
            }
            if (a.empty() || a[0] != '-') continue;
            auto need = [&](const char* opt) -> const char* {
                if (i + 1 >= argc) return nullptr;
                (void)opt;
                return argv[++i];
            };
            if (a == "-s") {
                const char* v = need("-s");
                if (!v) return fail("missing argument of -s option");
                char* end = nullptr;
                long id = std::strtol(v, &end, 10);
                if (end == v || id >= upbp_host::predefined_scene_count() || id < -1) return fail("invalid argument of -s option");
                if (id == 3 || id == 4 || id == 9 || id == 10) return fail("scenes 3, 4, 9, and 10 cannot be rendered with UPBP");
                c.scene_id = (int)id;
                if (id == -1) {
                    const char* f = need("-s");
                    if (!f) return fail("missing file name argument of -s option");
                    copy_str(c.scene_path, sizeof(c.scene_path), f);
                }
            } else if (a == "-a") {
                const char* v = need("-a");
                if (!v) return fail("missing argument of -a option");
                const std::string alg = v;
                if (alg == "upbp_all") {
                    c.algorithm_flags |= UPBP_BPT | UPBP_SURF | UPBP_PP3D | UPBP_PB2D | UPBP_BB1D;
                } else if (alg.size() >= 8 && alg.compare(0, 4, "upbp") == 0 && (alg[4] == '+' || alg[4] == '_')) {
                    c.algorithm_flags = 0;
                    if (alg[4] == '+') c.algorithm_flags |= UPBP_BPT | UPBP_SURF;
                    std::stringstream ss(alg.substr(5));
                    std::string t;
                    while (std::getline(ss, t, '+')) {
                        if (t == "bpt") c.algorithm_flags |= UPBP_BPT;
                        else if (t == "surf") c.algorithm_flags |= UPBP_SURF;
                        else if (t == "pp3d") c.algorithm_flags |= UPBP_PP3D;
                        else if (t == "pb2d") c.algorithm_flags |= UPBP_PB2D;
                        else if (t == "bb1d") c.algorithm_flags |= UPBP_BB1D;
                        else if (t == "bp2d") c.algorithm_flags |= UPBP_BP2D;
                        else return fail("invalid argument of -a option");
                    }
                }
            } else if (a == "-l") {
                const char* v = need("-l");
                if (!v) return fail("missing argument of -l option");
                char* end = nullptr;
                long l = std::strtol(v, &end, 10);
                if (end == v || l < 1) return fail("invalid argument of -l option");
                c.max_path_length = (uint32_t)l;
            } else if (a == "-t") {
                const char* v = need("-t");
                if (!v) return fail("missing argument of -t option");
                char* end = nullptr;
                double t = std::strtod(v, &end);
                if (end == v || t < 0) return fail("invalid argument of -t option");
                c.max_time = (float)t;
                extra << "_t" << v;
            } else if (a == "-i") {
                const char* v = need("-i");
                if (!v) return fail("missing argument of -i option");
                char* end = nullptr;
                long n = std::strtol(v, &end, 10);
                if (end == v || n < 1) return fail("invalid argument of -i option");
                c.iteration_count = (int)n;
            } else if (a == "-o") {
                const char* v = need("-o");
                if (!v || !*v) return fail("invalid argument of -o option");
                copy_str(c.output_name, sizeof(c.output_name), v);
            } else if (a == "-r") {
                const char* v = need("-r");
                if (!v) return fail("missing argument of -r option");
                int w = -1, h = -1;
                std::sscanf(v, "%dx%d", &w, &h);
                if (w <= 0 || h <= 0) return fail("invalid argument of -r option");
                c.res_x = (uint32_t)w;
                c.res_y = (uint32_t)h;
                extra << "_r" << v;
            } else if (a == "-r_alpha" || a == "-r_initial") {
                const bool is_alpha = a == "-r_alpha";
                const char* v = need(a.c_str());
                if (!v) return fail("missing argument of " + a + " option");
                float x = 0.f;
                std::sscanf(v, "%f", &x);
                if (is_alpha ? (x <= 0.f) : (x == 0.f)) return fail("invalid argument of " + a + " option");
                for (int k = 0; k < 5; k++) {
                    if (is_alpha && !set_alpha[k]) *alphas[k] = x;
                    if (!is_alpha && !set_init[k]) *inits[k] = x;
                }
                extra << (is_alpha ? "_ralpha" : "_rinit") << v;
            } else if (a.compare(0, 9, "-r_alpha_") == 0 || a.compare(0, 11, "-r_initial_") == 0) {
                const bool is_alpha = a.compare(0, 9, "-r_alpha_") == 0;
                const std::string tech = a.substr(is_alpha ? 9 : 11);
                int k = -1;
                for (int t = 0; t < 5; t++)
                    if (tech == tech_names[t]) k = t;
                if (k < 0) return fail("invalid option \"" + a + "\"");
                const char* v = need(a.c_str());
                if (!v) return fail("missing argument of " + a + " option");
                float x = 0.f;
                std::sscanf(v, "%f", &x);
                if (is_alpha ? (x <= 0.f) : (x == 0.f)) return fail("invalid argument of " + a + " option");
                if (is_alpha) {
                    *alphas[k] = x;
                    set_alpha[k] = true;
                    extra << "_ralpha" << tech << v;
                } else {
                    *inits[k] = x;
                    set_init[k] = true;
                    extra << "_rinit" << tech << v;
                }
            } else if (a == "-previous") {
                c.algorithm_flags |= UPBP_PREVIOUS;
                extra << "_prev";
            } else if (a == "-compatible") {
                c.algorithm_flags |= UPBP_COMPATIBLE;
                extra << "_comp";
            } else if (a == "-speconly") {
                c.algorithm_flags |= UPBP_SPECULAR_ONLY;
                extra << "_speconly";
            } else if (a == "-ignorespec") {
                const char* v = need("-ignorespec");
                if (!v) return fail("missing argument of -ignorespec option");
                if (std::string(v) == "1") c.ignore_fully_spec_paths = 1;
                else if (std::string(v) == "0") c.ignore_fully_spec_paths = 0;
                else return fail("invalid argument of -ignorespec option");
            } else if (a == "-qbt" || a == "-pbt") {
                const char* v = need(a.c_str());
                if (!v) return fail("missing argument of " + a + " option");
                const int t = (v[0] == 'L' || v[0] == 'l') ? UPBP_LONG_BEAM : UPBP_SHORT_BEAM;
                if (a == "-qbt") c.query_beam_type = t;
                else c.photon_beam_type = t;
            } else if (a == "-pbc") {
                const char* v = need("-pbc");
                if (!v) return fail("missing argument of -pbc option");
                float x = 0.f;
                std::sscanf(v, "%f", &x);
                if (x == 0.f) return fail("invalid argument of -pbc option");
                c.bb1d_used_light_subpath_count = x;
                extra << "_pbc" << v;
            } else if (a == "-continuous_output") {
                const char* v = need(a.c_str());
                if (!v) return fail("missing argument of -continuous_output option");
                char* end = nullptr;
                long n = std::strtol(v, &end, 10);
                if (end == v) return fail("invalid argument of -continuous_output option");
                c.continuous_output = (int)n;
            } else if (a == "-pcpi") {
                const char* v = need("-pcpi");
                if (!v) return fail("missing argument of -pcpi option");
                float x = 0.f;
                std::sscanf(v, "%f", &x);
                if (std::floor(x) == 0.f) return fail("invalid argument of -pcpi option");
                c.path_count_per_iter = x;
                extra << "_pcpi" << v;
            } else if (a == "-sn") {
                const char* v = need("-sn");
                if (!v) return fail("missing argument of -sn option");
                int x = 1;
                std::sscanf(v, "%d", &x);
                c.use_shading_normal = x == 0 ? 0 : 1;
                extra << "_sn" << v;
            } else if (a == "-assert") {
                c.gpu_assert = 1;
                extra << "_assert";
            } else if (a == "-ioff") {
                const char* v = need("-ioff");
                if (!v) return fail("missing argument of -ioff option");
                char* end = nullptr;
                long long n = std::strtoll(v, &end, 10);
                if (end == v || n < 0) return fail("invalid argument of -ioff option");
                c.iteration_offset = (uint64_t)n;
            } else if (a == "-log") {
                c.do_log = 1;
                extra << "_log";
            } else if (a == "-guide") {
                // not in the reference: learned proposal for scattering in media
                const char* v = need("-guide");
                if (!v) return fail("missing argument of -guide option");
                char* end = nullptr;
                const long n = std::strtol(v, &end, 10);
                if (end == v || n < 0) return fail("invalid argument of -guide option");
                c.guide_train_iterations = (int)n;
                extra << "_guide" << n;
            } else if (a == "-checkpoint" || a == "-resume") {
                // not in the reference: checkpoint / resume of a render
                const char* v = need(a.c_str());
                if (!v) return fail("missing argument of " + a + " option");
                if (std::strlen(v) >= sizeof(c.checkpoint_path)) return fail("path too long for " + a);
                std::snprintf(a == "-checkpoint" ? c.checkpoint_path : c.resume_path, sizeof(c.checkpoint_path),
                              "%s", v);
            } else if (a == "-mis_exact") {
                // not in the reference: full-path balance-heuristic weights
                // where the reference's recursion departs from them
                c.mis_exact = 1;
                extra << "_misexact";
            } else {
                return fail("invalid option \"" + a + "\"");
            }
        }
        if (c.path_count_per_iter < 0)
            c.path_count_per_iter = std::floor(-c.path_count_per_iter * (float)c.res_x * (float)c.res_y);
        else
            c.path_count_per_iter = std::floor(c.path_count_per_iter);
        if (c.output_name[0] == 0) {
            std::string name;
            if (c.scene_id > -1) {
                name = "s" + two_digits(c.scene_id);
            } else {
                const std::string p = c.scene_path;
                const size_t sl = p.find_last_of("\\/");
                const size_t dot = p.find_last_of('.');
                const size_t b = sl == std::string::npos ? 0 : sl + 1;
                name = "s-" + p.substr(b, dot == std::string::npos ? std::string::npos : dot - b);
            }
            copy_str(c.output_name, sizeof(c.output_name), name + default_suffix(c, extra.str()));
        }
        std::string on = c.output_name;
        const std::string ext = on.size() > 4 ? on.substr(on.size() - 4) : "";
        if (ext != ".bmp" && ext != ".exr") copy_str(c.output_name, sizeof(c.output_name), on + ".exr");
        *out = c;
        return UPBP_OK;
    });
}
