// terawarp -- command-line front end of libterawarp_b200 for the TeraWarp
// command (plugin_Bigimagewarp.cpp:73-107; README.md:85-100):
//
//   terawarp -i <img_sub> <marker_sub> <marker_tar> -o <out_dir> -p <params...> [options]
//
// -p takes either the plugin's seven strings, of which the reference reads
// the first three (program_mode device_mode downsample_mode;
// plugin_Bigimagewarp.cpp:78,91-93: program_mode 0 affine, 1 TPS), or the
// README's ten (warp_mode device_mode resize_mode deformation_mode para_x
// para_y para_z newsize_x newsize_y newsize_z).  <img_sub> is a .v3draw file
// or a directory of Z slices; results go to <out_dir> under the reference's
// names (<name>_stps.v3draw, <name>_affine_slice/, ... and _downsample
// previews), written by tw_bigimagewarp_files.
//
// Options beyond the reference's hard-coded values: --grid-spacing G (4),
// --interp linear|nn, --lambda L (0.2), --marker-scale S (1 for a file, 4 for a
// slice directory), --downsample 0|1, --gpu N (0).
//
// Exit status: 0 done, 1 the warp failed (the library's message is printed),
// 2 bad arguments.

#include "terawarp_b200.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

void usage(FILE *f)
{
    std::fprintf(f,
                 "usage: terawarp -i <img_sub> <marker_sub> <marker_tar> -o <out_dir> -p <params> [options]\n"
                 "  -p program_mode device_mode downsample_mode [4 more, ignored]\n"
                 "       program_mode 0 affine, 1 TPS; device_mode must be 1 (GPU)\n"
                 "  -p warp_mode device_mode resize_mode deformation_mode para_x para_y para_z\n"
                 "     newsize_x newsize_y newsize_z\n"
                 "       warp_mode 0 non-rigid (deformation 0 affine, 1 TPS, 2 scaling),\n"
                 "       1 rigid (deformation 0 rotation, 1 translation)\n"
                 "options: --grid-spacing G  --interp linear|nn  --lambda L  --marker-scale S\n"
                 "         --downsample 0|1  --gpu N\n");
}

bool parse_int(const char *s, long long &v)
{
    char *end = nullptr;
    v = std::strtoll(s, &end, 10);
    return end && end != s && *end == '\0';
}

bool parse_double(const char *s, double &v)
{
    char *end = nullptr;
    v = std::strtod(s, &end);
    return end && end != s && *end == '\0';
}

bool is_flag(const char *s) { return s[0] == '-' && (s[1] < '0' || s[1] > '9') && s[1] != '.'; }

}  // namespace

int main(int argc, char **argv)
{
    std::vector<std::string> in, out, par;
    int gpu = 0;
    tw_params p;
    tw_params_default(&p);
    p.marker_scale = 0.0;  // the plugin's choice per input: 1 for a .v3draw, 4 for a slice directory
    int downsample = -1;
    for (int a = 1; a < argc; ++a) {
        const char *s = argv[a];
        auto need = [&](int k) {
            if (a + k >= argc) {
                std::fprintf(stderr, "terawarp: %s needs a value\n", s);
                std::exit(2);
            }
        };
        if (!std::strcmp(s, "-h") || !std::strcmp(s, "--help")) {
            usage(stdout);
            return 0;
        } else if (!std::strcmp(s, "-i")) {
            while (a + 1 < argc && !is_flag(argv[a + 1])) in.push_back(argv[++a]);
        } else if (!std::strcmp(s, "-o")) {
            while (a + 1 < argc && !is_flag(argv[a + 1])) out.push_back(argv[++a]);
        } else if (!std::strcmp(s, "-p")) {
            while (a + 1 < argc && !is_flag(argv[a + 1])) par.push_back(argv[++a]);
        } else if (!std::strcmp(s, "--grid-spacing")) {
            need(1);
            long long g;
            if (!parse_int(argv[++a], g)) { std::fprintf(stderr, "terawarp: bad --grid-spacing\n"); return 2; }
            p.grid_spacing = (int)g;
        } else if (!std::strcmp(s, "--interp")) {
            need(1);
            const char *v = argv[++a];
            if (!std::strcmp(v, "linear")) p.interp = TW_INTERP_TRILINEAR;
            else if (!std::strcmp(v, "nn")) p.interp = TW_INTERP_NEAREST;
            else { std::fprintf(stderr, "terawarp: --interp is linear or nn\n"); return 2; }
        } else if (!std::strcmp(s, "--lambda")) {
            need(1);
            if (!parse_double(argv[++a], p.lambda)) { std::fprintf(stderr, "terawarp: bad --lambda\n"); return 2; }
        } else if (!std::strcmp(s, "--marker-scale")) {
            need(1);
            if (!parse_double(argv[++a], p.marker_scale)) { std::fprintf(stderr, "terawarp: bad --marker-scale\n"); return 2; }
        } else if (!std::strcmp(s, "--downsample")) {
            need(1);
            long long d;
            if (!parse_int(argv[++a], d) || (d != 0 && d != 1)) { std::fprintf(stderr, "terawarp: bad --downsample\n"); return 2; }
            downsample = (int)d;
        } else if (!std::strcmp(s, "--gpu")) {
            need(1);
            long long g;
            if (!parse_int(argv[++a], g) || g < 0) { std::fprintf(stderr, "terawarp: bad --gpu\n"); return 2; }
            gpu = (int)g;
        } else {
            std::fprintf(stderr, "terawarp: unknown argument %s\n", s);
            usage(stderr);
            return 2;
        }
    }
    if (in.size() != 3 || out.size() != 1) {
        std::fprintf(stderr, "terawarp: -i takes 3 paths and -o one\n");
        usage(stderr);
        return 2;
    }
    std::vector<double> v(par.size());
    for (size_t k = 0; k < par.size(); ++k)
        if (!parse_double(par[k].c_str(), v[k])) {
            std::fprintf(stderr, "terawarp: -p value %s is not a number\n", par[k].c_str());
            return 2;
        }
    if (par.size() == 7 || par.size() == 3) {
        // the plugin's form: program_mode device_mode downsample_mode
        const int program_mode = (int)v[0];
        if (program_mode != 0 && program_mode != 1) {
            std::fprintf(stderr, "terawarp: program_mode is 0 (affine) or 1 (TPS)\n");
            return 2;
        }
        p.warp_mode = 0;
        p.deformation_mode = program_mode;
        p.device_mode = (int)v[1];
        p.downsample_mode = (int)v[2];
    } else if (par.size() == 10) {
        p.warp_mode = (int)v[0];
        p.device_mode = (int)v[1];
        p.resize_mode = (int)v[2];
        p.deformation_mode = (int)v[3];
        p.para_x = v[4];
        p.para_y = v[5];
        p.para_z = v[6];
        p.newsize_x = (int64_t)v[7];
        p.newsize_y = (int64_t)v[8];
        p.newsize_z = (int64_t)v[9];
    } else {
        std::fprintf(stderr, "terawarp: -p takes 7 (or 3) or 10 values, got %zu\n", par.size());
        usage(stderr);
        return 2;
    }
    if (downsample >= 0) p.downsample_mode = downsample;

    tw_ctx *ctx = nullptr;
    tw_status st = tw_ctx_create(gpu, 0, &ctx);
    if (st != TW_OK) {
        std::fprintf(stderr, "terawarp: no GPU context on device %d: %s\n", gpu, tw_status_string(st));
        return 1;
    }
    st = tw_bigimagewarp_files(ctx, &p, in[0].c_str(), in[1].c_str(), in[2].c_str(), out[0].c_str());
    if (st != TW_OK) {
        std::fprintf(stderr, "terawarp: %s: %s\n", tw_status_string(st), tw_ctx_last_error(ctx));
        tw_ctx_destroy(ctx);
        return 1;
    }
    tw_ctx_destroy(ctx);
    std::printf("terawarp: done, results in %s\n", out[0].c_str());
    return 0;
}
