// `upbp` executable: the reference's main (gpuupbp/gpuupbp.cpp:57-148) on the
// C ABI: parse the command line, load the scene, run the iteration or time
// loop with optional continuous output, average and write the image.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/upbp.h"

// The reference saves with gamma 2.2 (framebuffer.hpp:66-70); the writer
// follows the name's extension (exr, bmp or hdr).
static int save_image(const std::string& name, const std::vector<float>& rgb, uint32_t w, uint32_t h)
{
    const int rc = upbp_write_image(name.c_str(), rgb.data(), w, h, 2.2f);
    if (rc != UPBP_OK) std::fprintf(stderr, "%s: %s\n", name.c_str(), upbp_last_error());
    return rc;
}

// -log: one CSV row per iteration in <timestamp>_log.txt, the reference's
// columns (misc/logger.cpp:32-86: scene, iter, light/build/camera time in
// seconds, resolution, device memory used/free/total in MiB, core
// utilisation -- 0, as the reference's without DBG_CORE_UTIL) and two more:
// subpaths per second and range queries per second of the iteration.
struct CsvLog {
    FILE* f = nullptr;
    explicit CsvLog(bool on)
    {
        if (!on) return;
        char stamp[80];
        const std::time_t t = std::time(nullptr);
        std::strftime(stamp, sizeof(stamp), "%Y-%m-%d-%H-%M-%S", std::localtime(&t));
        f = std::fopen((std::string(stamp) + "_log.txt").c_str(), "w");
        if (f)
            std::fprintf(f, "%40s,%6s,%12s,%12s,%12s,%12s,%12s,%12s,%12s,%12s,%12s,%12s,%12s,%12s\n", "scene", "iter",
                         "lighttime", "buildtime", "cameratime", "res_x", "res_y", "mem_used", "mem_free", "mem_total",
                         "light_util", "camera_util", "paths_per_s", "queries_per_s");
    }
    void row(const char* scene, int iter, upbp_ctx* ctx, uint32_t w, uint32_t h)
    {
        if (!f) return;
        upbp_stats st;
        if (upbp_get_stats(ctx, &st) != UPBP_OK) return;
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        const double mfree = fr / 1048576.0, mtot = tot / 1048576.0;
        const double s = (st.ms_light + st.ms_build + st.ms_camera) * 1e-3;
        const double paths = (double)st.light_paths + st.camera_paths;
        const double queries = (double)st.segment_queries + st.point_queries;
        std::fprintf(f, "%40s,%6d,%12g,%12g,%12g,%12u,%12u,%12g,%12g,%12g,%12g,%12g,%12g,%12g\n", scene, iter,
                     st.ms_light * 1e-3, st.ms_build * 1e-3, st.ms_camera * 1e-3, w, h, mtot - mfree, mfree, mtot,
                     0.0, 0.0, s > 0 ? paths / s : 0.0, s > 0 ? queries / s : 0.0);
        std::fflush(f);
    }
    ~CsvLog()
    {
        if (f) std::fclose(f);
    }
};

int main(int argc, const char** argv)
{
    upbp_config cfg;
    const int rc = upbp_parse_command_line(argc, argv, &cfg);
    if (rc != UPBP_OK) return rc == UPBP_HELP ? 0 : 1;
    upbp_scene* scene = nullptr;
    const int lrc = cfg.scene_id < 0 ? upbp_scene_load_obj(cfg.scene_path, cfg.res_x, cfg.res_y, &scene)
                                     : upbp_scene_load_predefined(cfg.scene_id, cfg.res_x, cfg.res_y, &scene);
    if (lrc != UPBP_OK) {
        std::fprintf(stderr, "scene: %s\n", upbp_last_error());
        return 1;
    }
    std::printf("Scene:    %s\n", cfg.scene_path);
    if (cfg.max_time > 0)
        std::printf("Target:   %g seconds render time\n", cfg.max_time);
    else
        std::printf("Target:   %d iteration(s)\n", cfg.iteration_count);
    upbp_ctx* ctx = nullptr;
    if (upbp_create(upbp_scene_get_desc(scene), &cfg, &ctx) != UPBP_OK) {
        std::fprintf(stderr, "init: %s\n", upbp_last_error());
        upbp_scene_free(scene);
        return 1;
    }
    int start = 0;  // iterations rendered before this run (a resumed checkpoint's)
    if (cfg.resume_path[0]) {
        if (upbp_load_checkpoint(ctx, cfg.resume_path) != UPBP_OK) {
            std::fprintf(stderr, "resume: %s\n", upbp_last_error());
            upbp_destroy(ctx);
            upbp_scene_free(scene);
            return 1;
        }
        upbp_stats st;
        if (upbp_get_stats(ctx, &st) == UPBP_OK) start = (int)st.iterations_done;
        std::printf("Resumed:  %d iteration(s) from %s\n", start, cfg.resume_path);
    }
    auto checkpoint = [&]() {
        if (cfg.checkpoint_path[0] && upbp_save_checkpoint(ctx, cfg.checkpoint_path) != UPBP_OK)
            std::fprintf(stderr, "checkpoint: %s\n", upbp_last_error());
    };
    const uint32_t w = cfg.res_x, h = cfg.res_y;
    const std::string out = cfg.output_name;
    const std::string stem = out.substr(0, out.size() - 4), ext = out.substr(out.size() - 3);
    CsvLog log(cfg.do_log != 0);
    auto t0 = std::chrono::steady_clock::now();
    int iter = start;
    auto continuous = [&](int done) {
        if (cfg.continuous_output > 0 && done % cfg.continuous_output == 0) {
            checkpoint();
            std::vector<float> img((size_t)w * h * 3, 0.f);
            upbp_accumulate_to_host(ctx, img.data(), 1.0 / done);
            char name[2048];
            std::snprintf(name, sizeof(name), "%s-%d.%s", stem.c_str(), done, ext.c_str());
            save_image(name, img, w, h);
        }
    };
    if (cfg.max_time > 0) {
        for (;;) {
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (el >= cfg.max_time) break;
            if (upbp_run_iteration(ctx, iter) < 0) break;  // > 0: status bits, the image is complete
            log.row(cfg.scene_path, iter, ctx, w, h);
            iter++;
            continuous(iter);
        }
    } else {
        int percent = -1;
        for (iter = start; iter < cfg.iteration_count; iter++) {
            if (upbp_run_iteration(ctx, iter) < 0) {  // > 0: status bits, the image is complete
                std::fprintf(stderr, "iteration %d: %s\n", iter, upbp_last_error());
                break;
            }
            log.row(cfg.scene_path, iter, ctx, w, h);
            const int p = (int)((float)(iter + 1) / cfg.iteration_count * 100.f);
            if (p != percent) {
                percent = p;
                std::printf("%d%%\n", p);
            }
            continuous(iter + 1);
        }
    }
    checkpoint();
    std::vector<float> img((size_t)w * h * 3, 0.f);
    upbp_accumulate_to_host(ctx, img.data(), iter > 0 ? 1.0 / iter : 0.0);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("done in %.2f s (%i iterations)\n", secs, iter);
    const int src = save_image(out, img, w, h);
    upbp_destroy(ctx);
    upbp_scene_free(scene);
    return src == UPBP_OK ? 0 : 1;
}
